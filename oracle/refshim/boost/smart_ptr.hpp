// Stand-in for boost/smart_ptr.hpp: std smart pointers under boost names.
#pragma once
#include <memory>
namespace boost {
using std::make_shared;
using std::shared_ptr;
template <class T>
class scoped_ptr {
 public:
  explicit scoped_ptr(T* p = nullptr) : p_(p) {}
  scoped_ptr(const scoped_ptr&) = delete;
  scoped_ptr& operator=(const scoped_ptr&) = delete;
  void reset(T* p = nullptr) { p_.reset(p); }
  T* get() const { return p_.get(); }
  T* operator->() const { return p_.get(); }
  T& operator*() const { return *p_; }

 private:
  std::unique_ptr<T> p_;
};
}  // namespace boost
