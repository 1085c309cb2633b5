// Stand-in for boost::alignment::aligned_allocator (test infrastructure).
// The reference uses it only to get 32-byte aligned std::vector<float> storage
// for its AVX2 loads (src/Constants.hpp:16-18).
#pragma once
#include <cstddef>
#include <cstdlib>
#include <new>

namespace boost {
namespace alignment {

template <class T, std::size_t Alignment = alignof(T)>
class aligned_allocator {
public:
    using value_type = T;
    template <class U>
    struct rebind {
        using other = aligned_allocator<U, Alignment>;
    };
    aligned_allocator() noexcept = default;
    template <class U>
    aligned_allocator(const aligned_allocator<U, Alignment>&) noexcept {}

    T* allocate(std::size_t n) {
        std::size_t a = Alignment < alignof(T) ? alignof(T) : Alignment;
        std::size_t bytes = n * sizeof(T);
        bytes = (bytes + a - 1) / a * a;
        if (bytes == 0) bytes = a;
        void* p = std::aligned_alloc(a, bytes);
        if (!p) throw std::bad_alloc();
        return static_cast<T*>(p);
    }
    void deallocate(T* p, std::size_t) noexcept { std::free(p); }

    template <class U>
    bool operator==(const aligned_allocator<U, Alignment>&) const noexcept { return true; }
    template <class U>
    bool operator!=(const aligned_allocator<U, Alignment>&) const noexcept { return false; }
};

}  // namespace alignment
}  // namespace boost
