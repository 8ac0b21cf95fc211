// Replacement for the reference's Threading/Atomic.h, found first on the
// include path when the engine headers are compiled here (the GPU space plug-in
// and the CPU checker built from the reference sources).
//
// Why: on GCC the reference's AtomicInt32::Exchange / AtomicInt64::Exchange
// (Core/Threading/Atomic.h:200-212 and :395-405) loop while the CAS
// *succeeds*, so they never return, and every List<T>::Clear()
// (Core/Threading/List.h:384) hangs. List<T>::PopBack (List.h:423) also calls
// AtomicInt32::Decrement on a size_t. This header provides the same class
// names and static entry points over the GCC __atomic builtins with a
// terminating exchange and a size_t decrement. None of it is on the traced
// arithmetic path; it only makes the reference's containers usable.
#pragma once

#include <utility>
#include <string>
#include <sstream>
#include <cstddef>

#include <boost/format.hpp>

#include "System/Platform.h"

namespace Illumina
{
	namespace Core
	{
		class AtomicInt32
		{
		private:
			volatile Int32 m_int32;

		public:
			AtomicInt32(Int32 v) : m_int32(v) { }
			AtomicInt32(const AtomicInt32 &o) : m_int32(o.m_int32) { }

			Int32 operator++(void) { return __atomic_add_fetch(&m_int32, 1, __ATOMIC_SEQ_CST); }
			Int32 operator++(int) { return __atomic_fetch_add(&m_int32, 1, __ATOMIC_SEQ_CST); }
			Int32 operator--(void) { return __atomic_sub_fetch(&m_int32, 1, __ATOMIC_SEQ_CST); }
			Int32 operator--(int) { return __atomic_fetch_sub(&m_int32, 1, __ATOMIC_SEQ_CST); }
			Int32 operator+=(Int32 v) { return __atomic_add_fetch(&m_int32, v, __ATOMIC_SEQ_CST); }
			Int32 operator-=(Int32 v) { return __atomic_sub_fetch(&m_int32, v, __ATOMIC_SEQ_CST); }
			Int32 operator=(Int32 v) { __atomic_store_n(&m_int32, v, __ATOMIC_SEQ_CST); return v; }
			operator long(void) { return (long)__atomic_load_n(&m_int32, __ATOMIC_SEQ_CST); }

			static inline Int32 Add(Int32 *p, Int32 v) { return __atomic_add_fetch(p, v, __ATOMIC_SEQ_CST); }
			static inline Int32 Increment(Int32 *p) { return __atomic_add_fetch(p, 1, __ATOMIC_SEQ_CST); }
			static inline Int32 Decrement(Int32 *p) { return __atomic_sub_fetch(p, 1, __ATOMIC_SEQ_CST); }
			static inline size_t Decrement(size_t *p) { return __atomic_sub_fetch(p, (size_t)1, __ATOMIC_SEQ_CST); }
			static inline Int32 Exchange(Int32 *p, Int32 v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }
			static inline Int32 FetchAndAdd(Int32 *p, Int32 v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
			static inline Int32 CompareAndSwap(Int32 *p, Int32 xchg, Int32 cmp) { return __sync_val_compare_and_swap(p, cmp, xchg); }

			std::string ToString(void) const { std::ostringstream s; s << m_int32; return s.str(); }
		};

		class AtomicInt64
		{
		private:
			volatile Int64 m_int64;

		public:
			AtomicInt64(Int64 v) : m_int64(v) { }
			AtomicInt64(const AtomicInt64 &o) : m_int64(o.m_int64) { }

			Int64 operator++(void) { return __atomic_add_fetch(&m_int64, 1, __ATOMIC_SEQ_CST); }
			Int64 operator++(int) { return __atomic_fetch_add(&m_int64, 1, __ATOMIC_SEQ_CST); }
			Int64 operator--(void) { return __atomic_sub_fetch(&m_int64, 1, __ATOMIC_SEQ_CST); }
			Int64 operator--(int) { return __atomic_fetch_sub(&m_int64, 1, __ATOMIC_SEQ_CST); }
			operator long long(void) { return (long long)__atomic_load_n(&m_int64, __ATOMIC_SEQ_CST); }

			static inline Int64 Add(Int64 *p, Int64 v) { return __atomic_add_fetch(p, v, __ATOMIC_SEQ_CST); }
			static inline Int64 Increment(Int64 *p) { return __atomic_add_fetch(p, 1, __ATOMIC_SEQ_CST); }
			static inline Int64 Decrement(Int64 *p) { return __atomic_sub_fetch(p, 1, __ATOMIC_SEQ_CST); }
			static inline Int64 Exchange(Int64 *p, Int64 v) { return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST); }
			static inline Int64 FetchAndAdd(Int64 *p, Int64 v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
			static inline Int64 CompareAndSwap(Int64 *p, Int64 xchg, Int64 cmp) { return __sync_val_compare_and_swap(p, cmp, xchg); }

			std::string ToString(void) const { std::ostringstream s; s << m_int64; return s.str(); }
		};
	}
}
