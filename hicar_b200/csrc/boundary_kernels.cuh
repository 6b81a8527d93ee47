// Lateral-boundary update and clipping for the advected species.
//   k_apply_forcing   apply_forcing, advected 3-D branch, src/objects/domain_obj.f90:3495-3506
//   k_enforce_limits  enforce_limits, src/objects/domain_obj.f90:3124-3147
#pragma once
#include "common.cuh"

namespace icar {

// Relaxation-zone update over the columns whose filter is non-zero (zone[]
// holds their (i,j) packed as i + nx*j), for every species that has forcing
// in one launch (thread index = (species slot, level, zone column)).  dt is
// the real64 dt%seconds(); the Fortran expression mixes real and real64, so
// it is evaluated in double and rounded on assignment.  Columns with filter
// 0 are left alone: the reference adds 0*(forcing-q) there, which leaves q
// unchanged for finite inputs.  Forcing values are advanced only inside the
// zone, the only place the advected species read them.
struct ForcingPtrs {
    float *q[32];
    float *forcing[32];
    const float *dqdt[32];
};

__global__ void k_apply_forcing(Geo g, int nzone, const int *__restrict__ zone,
                                const float *__restrict__ filter2d, double dt, ForcingPtrs fp, int nslots)
{
    const size_t per = (size_t)nzone * g.nz;
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= per * (size_t)nslots) return;
    const int s = (int)(t / per);
    const size_t r = t - (size_t)s * per;
    const int z = (int)(r % (size_t)nzone);
    const int k = (int)(r / (size_t)nzone);
    float *__restrict__ q = fp.q[s];
    float *__restrict__ forcing = fp.forcing[s];
    const int packed = zone[z];
    const int i = packed % g.nx, j = packed / g.nx;
    const size_t c = ix(g, i, k, j);
    const float fnew = (float)((double)forcing[c] + (double)fp.dqdt[s][c] * dt);
    forcing[c] = fnew;
    const float flt = filter2d[packed];
    if (flt == 1.0f)
        q[c] = fnew;
    else if (flt < 1.0f)
        q[c] = (float)((double)q[c] + ((double)flt * dt / 3600.0) * (double)(fnew - q[c]));
}

__global__ void k_enforce_limits(Geo g, float *__restrict__ q)
{
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    size_t n = (size_t)g.P * g.nz * g.ny;
    if (t >= n) return;
    if ((int)(t % (size_t)g.P) >= g.nx) return;
    float v = q[t];
    if (v < 0.0f) q[t] = 0.0f;
}

}  // namespace icar
