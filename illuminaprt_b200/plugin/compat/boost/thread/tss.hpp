#pragma once
namespace boost {
// Per-thread pointer slot (thread_local storage keyed by the slot object).
template <class T> class thread_specific_ptr {
  static thread_local T *slot_;
public:
  T *get() const { return slot_; }
  T *operator->() const { return slot_; }
  T &operator*() const { return *slot_; }
  void reset(T *p = 0) { delete slot_; slot_ = p; }
};
template <class T> thread_local T *thread_specific_ptr<T>::slot_ = 0;
}
