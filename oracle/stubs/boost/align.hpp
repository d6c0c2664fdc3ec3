/*
 * Stand-in for boost::alignment::aligned_allocator, used only to compile the
 * reference's hot-path sources into the CPU oracle (test infrastructure).
 */
#ifndef ORACLE_STUB_BOOST_ALIGN_HPP
#define ORACLE_STUB_BOOST_ALIGN_HPP

#include <cstddef>
#include <cstdlib>
#include <new>

namespace boost {
namespace alignment {

template <class T, std::size_t Alignment>
class aligned_allocator {
public:
    typedef T value_type;
    typedef T* pointer;
    typedef const T* const_pointer;
    typedef T& reference;
    typedef const T& const_reference;
    typedef std::size_t size_type;
    typedef std::ptrdiff_t difference_type;
    template <class U> struct rebind { typedef aligned_allocator<U, Alignment> other; };

    aligned_allocator() noexcept {}
    template <class U> aligned_allocator(const aligned_allocator<U, Alignment>&) noexcept {}

    T* allocate(std::size_t count) {
        std::size_t bytes = count * sizeof(T);
        std::size_t rounded = (bytes + Alignment - 1) / Alignment * Alignment;
        if (rounded == 0) rounded = Alignment;
        void* p = nullptr;
        if (posix_memalign(&p, Alignment < sizeof(void*) ? sizeof(void*) : Alignment, rounded) != 0)
            throw std::bad_alloc();
        return static_cast<T*>(p);
    }
    void deallocate(T* p, std::size_t) noexcept { std::free(p); }
};

template <class T, class U, std::size_t A>
bool operator==(const aligned_allocator<T, A>&, const aligned_allocator<U, A>&) noexcept { return true; }
template <class T, class U, std::size_t A>
bool operator!=(const aligned_allocator<T, A>&, const aligned_allocator<U, A>&) noexcept { return false; }

}  // namespace alignment
}  // namespace boost

#endif
