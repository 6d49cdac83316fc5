// hugevec.hpp -- std::vector backed by transparent huge pages.
//
// The host copies of a 100M-synapse network are several GB; with 4 KB pages
// their first touch costs millions of page faults.  Large blocks are
// 2 MB-aligned and advised MADV_HUGEPAGE instead.
#pragma once

#include <stdlib.h>
#include <sys/mman.h>

#include <new>
#include <vector>

namespace nemo_b200 {

template<typename T>
struct HugeAllocator {
	using value_type = T;
	static constexpr size_t HUGE = size_t(2) << 20;

	HugeAllocator() = default;
	template<typename U> HugeAllocator(const HugeAllocator<U>&) {}

	T* allocate(size_t n)
	{
		size_t bytes = n * sizeof(T);
		if(bytes < HUGE) {
			return static_cast<T*>(::operator new(bytes));
		}
		size_t len = (bytes + HUGE - 1) & ~(HUGE - 1);
		void* p = nullptr;
		if(posix_memalign(&p, HUGE, len) != 0) throw std::bad_alloc();
		madvise(p, len, MADV_HUGEPAGE);
		return static_cast<T*>(p);
	}

	void deallocate(T* p, size_t n)
	{
		if(n * sizeof(T) < HUGE) ::operator delete(p);
		else free(p);
	}

	template<typename U> bool operator==(const HugeAllocator<U>&) const { return true; }
	template<typename U> bool operator!=(const HugeAllocator<U>&) const { return false; }
};

template<typename T>
using hvector = std::vector<T, HugeAllocator<T>>;

} // namespace nemo_b200
