// Minimal host-only stand-in for the Umpire allocator API used by Devil Ray's
// Array registry.  Every allocator is plain malloc/free on the host; "copy"
// is memcpy using the size recorded at allocation.  Test-oracle use only.
#ifndef ORACLE_SHIM_UMPIRE_HPP
#define ORACLE_SHIM_UMPIRE_HPP

#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

namespace umpire
{
struct MemoryResourceTraits
{
  enum class resource_type { host, device, unknown };
  resource_type resource = resource_type::host;
};

struct AllocationStrategy
{
  MemoryResourceTraits traits;
  MemoryResourceTraits getTraits () const { return traits; }
};

class ResourceManager;

class Allocator
{
  friend class ResourceManager;
  int m_id = 0;
  AllocationStrategy *m_strategy = nullptr;

  public:
  Allocator () = default;
  void *allocate (std::size_t bytes);
  void deallocate (void *ptr);
  int getId () const { return m_id; }
  AllocationStrategy *getAllocationStrategy () const { return m_strategy; }
};

class ResourceManager
{
  std::mutex m_mutex;
  std::map<void *, std::size_t> m_sizes;
  AllocationStrategy m_host_strategy;
  AllocationStrategy m_device_strategy;

  ResourceManager ()
  {
    m_device_strategy.traits.resource = MemoryResourceTraits::resource_type::device;
  }

  public:
  static ResourceManager &getInstance ()
  {
    static ResourceManager rm;
    return rm;
  }

  Allocator getAllocator (const std::string &name)
  {
    Allocator a;
    a.m_id = (name == "DEVICE") ? 1 : 0;
    a.m_strategy = (name == "DEVICE") ? &m_device_strategy : &m_host_strategy;
    return a;
  }

  Allocator getAllocator (int id)
  {
    if (id < 0 || id > 3) throw std::runtime_error ("umpire shim: bad allocator id");
    Allocator a;
    a.m_id = id;
    a.m_strategy = (id == 1 || id == 3) ? &m_device_strategy : &m_host_strategy;
    return a;
  }

  template <typename Strategy, typename... Args>
  Allocator makeAllocator (const std::string &name, Allocator base, Args...)
  {
    Allocator a = base;
    a.m_id = base.m_id + 2;
    return a;
  }

  void *raw_allocate (std::size_t bytes)
  {
    void *p = std::malloc (bytes == 0 ? 1 : bytes);
    std::lock_guard<std::mutex> g (m_mutex);
    m_sizes[p] = bytes;
    return p;
  }

  void raw_deallocate (void *p)
  {
    {
      std::lock_guard<std::mutex> g (m_mutex);
      m_sizes.erase (p);
    }
    std::free (p);
  }

  void copy (void *dst, void *src)
  {
    std::size_t n = 0;
    {
      std::lock_guard<std::mutex> g (m_mutex);
      auto it = m_sizes.find (src);
      if (it != m_sizes.end ()) n = it->second;
    }
    if (n && dst != src) std::memcpy (dst, src, n);
  }
};

inline void *Allocator::allocate (std::size_t bytes)
{
  return ResourceManager::getInstance ().raw_allocate (bytes);
}
inline void Allocator::deallocate (void *ptr)
{
  ResourceManager::getInstance ().raw_deallocate (ptr);
}

} // namespace umpire

#endif
