// Single-element field inversion for the one-per-block inversions of the
// batch-invert and product kernels.  Binary extended Euclid on the residue
// (shifts and subtractions on the ALU pipes) has a much shorter dependent
// chain than Fermat's ~310 Montgomery products, which matters because a
// whole CTA waits on it.  The result is converted back to Montgomery form
// with two multiplications by R^2.  Inverse of zero is zero.
#pragma once
#include "field.cuh"

namespace h2b {

H2B_DEV void u256_shr1(uint32_t (&u)[8])
{
#pragma unroll
    for (int i = 0; i < 7; i++) u[i] = __funnelshift_r(u[i], u[i + 1], 1);
    u[7] >>= 1;
}

// d = a - b; returns true on borrow (a < b).
H2B_DEV bool u256_sub(uint32_t (&d)[8], const uint32_t (&a)[8], const uint32_t (&b)[8])
{
    uint32_t bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]), "=r"(bw)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(b[0]),
          "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
    return bw != 0;
}

template <class C>
H2B_DEV void half_mod(uint32_t (&x)[8])
{
    if (x[0] & 1u) {
        // x + m < 2^255: no carry out of the top word
        const uint32_t m[8] = {C::M0, C::M1, C::M2, C::M3, C::M4, C::M5, C::M6, C::M7};
        asm("add.cc.u32  %0, %0, %8;\n\t"
            "addc.cc.u32 %1, %1, %9;\n\t"
            "addc.cc.u32 %2, %2, %10;\n\t"
            "addc.cc.u32 %3, %3, %11;\n\t"
            "addc.cc.u32 %4, %4, %12;\n\t"
            "addc.cc.u32 %5, %5, %13;\n\t"
            "addc.cc.u32 %6, %6, %14;\n\t"
            "addc.u32    %7, %7, %15;"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7])
            : "r"(m[0]), "r"(m[1]), "r"(m[2]), "r"(m[3]), "r"(m[4]), "r"(m[5]), "r"(m[6]), "r"(m[7]));
    }
    u256_shr1(x);
}

H2B_DEV bool u256_is_one(const uint32_t (&u)[8])
{
    return u[0] == 1u && (u[1] | u[2] | u[3] | u[4] | u[5] | u[6] | u[7]) == 0u;
}

H2B_DEV bool u256_is_zero(const uint32_t (&u)[8])
{
    return (u[0] | u[1] | u[2] | u[3] | u[4] | u[5] | u[6] | u[7]) == 0u;
}

template <class C>
H2B_DEV Fp<C> finv_fast(const Fp<C>& a)
{
    if (a.is_zero()) return a;
    uint32_t u[8], v[8];
    Fp<C> x1 = Fp<C>::zero(), x2 = Fp<C>::zero();
    x1.v[0] = 1u;
#pragma unroll
    for (int i = 0; i < 8; i++) u[i] = a.v[i];
    v[0] = C::M0; v[1] = C::M1; v[2] = C::M2; v[3] = C::M3;
    v[4] = C::M4; v[5] = C::M5; v[6] = C::M6; v[7] = C::M7;
    // invariants: x1 * a == u, x2 * a == v (mod m), as plain residues.
    // For a canonical nonzero a the loop ends within ~2*256 halvings and 512
    // subtractions; the caps only stop a non-canonical input (a multiple of
    // m) from spinning -- it then returns zero like the zero input.
    int guard = 0;
#pragma unroll 1
    while (!u256_is_one(u) && !u256_is_one(v)) {
        if (++guard > 2048 || u256_is_zero(u) || u256_is_zero(v)) return Fp<C>::zero();
#pragma unroll 1
        while ((u[0] & 1u) == 0u) { u256_shr1(u); half_mod<C>(x1.v); }
#pragma unroll 1
        while ((v[0] & 1u) == 0u) { u256_shr1(v); half_mod<C>(x2.v); }
        uint32_t d[8];
        if (!u256_sub(d, u, v)) {
#pragma unroll
            for (int i = 0; i < 8; i++) u[i] = d[i];
            x1 = x1 - x2;
        } else {
            u256_sub(d, v, u);
#pragma unroll
            for (int i = 0; i < 8; i++) v[i] = d[i];
            x2 = x2 - x1;
        }
    }
    Fp<C> r = u256_is_one(u) ? x1 : x2;   // r = (aR)^-1 as a plain residue = a^-1 R^-1
    r = r * Fp<C>::r2();                  // a^-1
    return r * Fp<C>::r2();               // a^-1 R  (Montgomery form)
}

} // namespace h2b
