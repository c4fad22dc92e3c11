// Vectors of plain data whose resize leaves the new elements default-initialised (no zero
// fill): for the set-up arrays whose every element the construction writes before anything
// reads it, so those writes (in parallel) are the arrays' first touch.
#pragma once
#include <memory>
#include <type_traits>
#include <utility>
#include <vector>

namespace gpl {

template <class T>
struct DefaultInitAlloc : std::allocator<T> {
  using value_type = T;
  template <class U>
  struct rebind {
    using other = DefaultInitAlloc<U>;
  };
  DefaultInitAlloc() = default;
  template <class U>
  DefaultInitAlloc(const DefaultInitAlloc<U> &) noexcept {}
  template <class U>
  void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new ((void *)p) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new ((void *)p) U(std::forward<A>(a)...);
  }
};
template <class T>
using pod_vector = std::vector<T, DefaultInitAlloc<T>>;

}  // namespace gpl
