#pragma once
#include <cstdint>
namespace boost { namespace interprocess { namespace ipcdetail {
inline uint32_t atomic_inc32(volatile uint32_t *m) { return __sync_fetch_and_add(m, 1u); }
inline uint32_t atomic_dec32(volatile uint32_t *m) { return __sync_fetch_and_sub(m, 1u); }
inline void atomic_write32(volatile uint32_t *m, uint32_t v) { __sync_lock_test_and_set(m, v); }
inline uint32_t atomic_cas32(volatile uint32_t *m, uint32_t with, uint32_t cmp) { return __sync_val_compare_and_swap(m, cmp, with); }
} } }
