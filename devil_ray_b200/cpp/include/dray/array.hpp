// dray::Array<T> for the B200 path: a reference-counted buffer with a host
// copy and a device copy kept coherent lazily, like the reference's Array
// (array.hpp:19-41, array_internals.hpp:174-215): copies share storage,
// asking for one side's pointer brings that side up to date, and asking
// for a writable pointer marks the other side stale.  Device memory comes
// from cudaMalloc; there is no CPU fallback for the kernels that use it.
#pragma once

#include <cstddef>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

namespace dray
{

typedef int int32;
typedef unsigned int uint32;
typedef long long int int64;
typedef float float32;
typedef double float64;
typedef float Float;

class DRayError : public std::runtime_error
{
  public:
  explicit DRayError (const std::string &msg) : std::runtime_error (msg) {}
  std::string GetMessage () const { return what (); }
};

#define DRAY_ERROR(msg)                                                                  \
  do                                                                                     \
  {                                                                                      \
    std::ostringstream drb_oss__;                                                        \
    drb_oss__ << msg << " (" << __FILE__ << ":" << __LINE__ << ")";                      \
    throw ::dray::DRayError (drb_oss__.str ());                                          \
  } while (0)

inline void cuda_check (cudaError_t e, const char *what)
{
  if (e != cudaSuccess) throw DRayError (std::string (what) + ": " + cudaGetErrorString (e));
}

template <typename T> class Array
{
  struct Store
  {
    T *host = nullptr;
    T *device = nullptr;
    size_t size = 0;
    bool host_valid = true;    // host copy holds the latest data
    bool device_valid = true;  // device copy holds the latest data
    ~Store ()
    {
      delete[] host;
      if (device) cudaFree (device);
    }
  };
  std::shared_ptr<Store> m_s;

  void ensure_host () const
  {
    Store &s = *m_s;
    if (!s.host && s.size) s.host = new T[s.size];
    if (!s.host_valid && s.size)
    {
      cuda_check (cudaMemcpy (s.host, s.device, sizeof (T) * s.size, cudaMemcpyDeviceToHost),
                  "Array: device to host copy");
    }
    s.host_valid = true;
  }
  void ensure_device () const
  {
    Store &s = *m_s;
    if (!s.device && s.size)
      cuda_check (cudaMalloc ((void **)&s.device, sizeof (T) * s.size), "Array: cudaMalloc");
    if (!s.device_valid && s.size)
    {
      cuda_check (cudaMemcpy (s.device, s.host, sizeof (T) * s.size, cudaMemcpyHostToDevice),
                  "Array: host to device copy");
    }
    s.device_valid = true;
  }

  public:
  Array () : m_s (std::make_shared<Store> ()) {}
  Array (const T *data, size_t n) : Array () { set (data, n); }

  size_t size () const { return m_s->size; }

  // New storage of n elements with undefined contents: both sides count as
  // current, so the first writer (host or device) copies nothing.
  void resize (size_t n)
  {
    if (n == m_s->size) return;
    auto s = std::make_shared<Store> ();
    s->size = n;
    m_s = s;
  }

  void set (const T *data, size_t n)
  {
    resize (n);
    if (n) std::memcpy (get_host_ptr (), data, sizeof (T) * n);
  }

  T *get_host_ptr ()
  {
    ensure_host ();
    m_s->device_valid = false;
    return m_s->host;
  }
  const T *get_host_ptr_const () const
  {
    ensure_host ();
    return m_s->host;
  }
  T *get_device_ptr ()
  {
    ensure_device ();
    m_s->host_valid = false;
    return m_s->device;
  }
  const T *get_device_ptr_const () const
  {
    ensure_device ();
    return m_s->device;
  }
};

} // namespace dray
