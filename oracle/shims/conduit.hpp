// Inert host-only stand-in for conduit::Node, enough for Devil Ray's
// to_node()/from_node() members to compile.  The oracle never serialises
// through it.  Test-oracle use only.
#ifndef ORACLE_SHIM_CONDUIT_HPP
#define ORACLE_SHIM_CONDUIT_HPP

#include <cstdint>
#include <map>
#include <memory>
#include <string>

namespace conduit
{
class DataType
{
  long long m_n = 0;
  public:
  DataType () = default;
  explicit DataType (long long n) : m_n (n) {}
  bool is_empty () const { return m_n == 0; }
  long long number_of_elements () const { return m_n; }
};

class Node
{
  std::map<std::string, std::shared_ptr<Node>> m_children;
  const void *m_ptr = nullptr;
  long long m_n = 0;
  long long m_int = 0;

  public:
  Node () = default;
  Node &operator[] (const std::string &path)
  {
    auto &c = m_children[path];
    if (!c) c = std::make_shared<Node> ();
    return *c;
  }
  const Node &operator[] (const std::string &path) const
  {
    static const Node empty;
    auto it = m_children.find (path);
    return it == m_children.end () ? empty : *it->second;
  }
  bool has_path (const std::string &path) const
  {
    return m_children.count (path) != 0;
  }
  void reset ()
  {
    m_children.clear ();
    m_ptr = nullptr;
    m_n = 0;
    m_int = 0;
  }
  template <typename T> void set_external (T *ptr, long long n)
  {
    m_ptr = ptr;
    m_n = n;
  }
  Node &operator= (int v) { m_int = v; m_n = 1; return *this; }
  Node &operator= (long v) { m_int = v; m_n = 1; return *this; }
  Node &operator= (long long v) { m_int = v; m_n = 1; return *this; }
  Node &operator= (unsigned v) { m_int = v; m_n = 1; return *this; }
  Node &operator= (unsigned long v) { m_int = (long long)v; m_n = 1; return *this; }
  Node &operator= (unsigned long long v) { m_int = (long long)v; m_n = 1; return *this; }
  Node &operator= (float v) { m_int = (long long)v; m_n = 1; return *this; }
  Node &operator= (double v) { m_int = (long long)v; m_n = 1; return *this; }
  Node &operator= (const std::string &) { m_n = 1; return *this; }
  Node &operator= (const char *) { m_n = 1; return *this; }
  int32_t to_int32 () const { return (int32_t)m_int; }
  int32_t to_int () const { return (int32_t)m_int; }
  DataType dtype () const { return DataType (m_n); }
  const float *as_float32_ptr () const { return (const float *)m_ptr; }
  const double *as_float64_ptr () const { return (const double *)m_ptr; }
  const int32_t *as_int32_ptr () const { return (const int32_t *)m_ptr; }
};
} // namespace conduit

#endif
