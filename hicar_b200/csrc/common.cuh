// Shared device helpers for the advection kernels.
//
// Arithmetic contract: every kernel evaluates the reference's Fortran
// expressions in the same order, with IEEE-rounded division and with
// multiply-add fusion disabled (the library is compiled with -fmad=false), so
// results match the CPU restatement bit for bit.  min/max/abs follow the
// C ternary forms the restatement uses, which keeps signed zeros identical.
#pragma once
#include <cstddef>
#include <cstdint>

namespace icar {

// Geometry of one resident domain.  Every 3-D array uses the row pitch P
// (elements, >= nx+1, multiple of 4 so rows start on 16-byte boundaries):
// element (i,k,j) sits at i + P*(k + nz*j).  Cell fields use i < nx; x-face
// fields use i <= nx (face i between cells i-1 and i); y-face fields have
// ny+1 rows (face j between rows j-1 and j); z-face fields store the top face
// of cell k at level k.
struct Geo {
    int nx, ny, nz, P;
};

__host__ __device__ __forceinline__ size_t ix(const Geo &g, int i, int k, int j)
{
    return (size_t)i + (size_t)g.P * ((size_t)k + (size_t)g.nz * (size_t)j);
}

__device__ __forceinline__ float fmax_(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float fmin_(float a, float b) { return a < b ? a : b; }

// Donor-cell flux, src/physics/adv_mpdata.f90:23-41.
__device__ __forceinline__ float flux1(float l, float r, float U)
{
    float a = fabsf(U);
    return ((U + a) * l + (U - a) * r) / 2.0f;
}

}  // namespace icar
