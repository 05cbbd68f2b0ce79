/*
 * oracle/shim/shim_alloc.cpp -- zero-filling global operator new for the
 * checker binary oracle/_ref/BECMPI_ref.  TEST INFRASTRUCTURE ONLY.
 *
 * With one rank the reference scatters one particle past the end of each IC
 * chunk's position/velocity vectors (src/gadget_IC.h:431-432 sets
 * numpart_per_rank[last] = numpart - sum + 1; src/gadget_IC.h:500-510 copies
 * that many).  The read stays inside the vector's capacity (3*npart is never
 * a power of two, libstdc++ grows capacity in powers of two) but the bytes
 * there are otherwise indeterminate.  Zero-filling every allocation makes
 * that "phantom" particle deterministically sit at the origin with zero
 * velocity, which is what the product's IFDM_IC_REF1 compatibility mode
 * reproduces.
 */
#include <cstdlib>
#include <new>

void *operator new(std::size_t n) {
    void *p = std::calloc(n ? n : 1, 1);
    if (!p) throw std::bad_alloc();
    return p;
}
void *operator new[](std::size_t n) { return operator new(n); }
void operator delete(void *p) noexcept { std::free(p); }
void operator delete[](void *p) noexcept { std::free(p); }
void operator delete(void *p, std::size_t) noexcept { std::free(p); }
void operator delete[](void *p, std::size_t) noexcept { std::free(p); }
