// libicar_adv: C ABI (include/icar_adv.h) over the sm_100a advection kernels.
//
// A handle (icar_adv_domain) is the device-resident image of one ICAR
// domain_t: species, winds and metric fields live in HBM with a common row
// pitch; the host only moves data on explicit set/get calls.  Work is
// enqueued on the handle's stream; failures are returned as status codes with
// a message, never by aborting.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <mutex>
#include <thread>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/icar_adv.h"
#include "boundary_kernels.cuh"
#include "common.cuh"
#include "mpdata_fused.cuh"
#include "mpdata_kernels.cuh"
#include "std_kernels.cuh"
#include "std_fused.cuh"
#include "batch_kernels.cuh"
#include "wind_kernels.cuh"
#include "mp_kernels.cuh"
#include "mpdata_onepass.cuh"

using icar::Geo;

namespace {

thread_local std::string g_create_error;

struct DevBuf {
    float *p = nullptr;
    size_t n = 0;  // elements
};

}  // namespace

struct icar_adv_domain {
    icar_adv_desc desc{};
    icar_adv_opts opts{};
    int hs = 2;
    Geo g{};
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    // icar_adv_step_host: copy streams and per-group events, created on first use
    cudaStream_t io_in = nullptr, io_out = nullptr;
    std::vector<cudaEvent_t> io_events;
    size_t n_cell = 0, n_u = 0, n_v = 0, n_zf = 0;
    size_t bytes = 0;
    // resident inputs
    DevBuf u, v, w, rho, jac, jac_u, jac_v, jac_w, dz;
    bool have_u = false, have_v = false, have_w = false, have_rho = false, have_jac = false,
         have_jac_u = false, have_jac_v = false, have_jac_w = false, have_dz = false;
    std::vector<DevBuf> q;           // species, adv_vars order
    std::vector<bool> have_q;
    std::vector<DevBuf> forcing, dqdt;
    DevBuf spare;                    // output buffer of the fused kernel (swapped with a species)
    // relaxation zone
    std::vector<float> filter_host;  // nx*ny
    float *filter_dev = nullptr;
    int *zone_dev = nullptr;
    int nzone = 0;
    // per-step Courant fluxes and staged-path scratch
    DevBuf Um, Vm, Wm;
    DevBuf q1, u2, v2, w2, u2l, v2l, w2l;      // MPDATA staged scratch
    DevBuf Gc, DJR, Wp;                        // fused path: J*rho, dz*J*rho, W_m/dz
    DevBuf dtbuf;                              // compute_dt: 4 maxima then dz_levels (nz)
    // simple microphysics: its extra resident fields, the real64 rain and
    // snow accumulations (nx*ny each) and the device stop flag
    DevBuf pressure, exner, dz_mass;
    bool have_pressure = false, have_exner = false, have_dz_mass = false;
    DevBuf dz_interface;                      // kept for restarts only (the path does not read it)
    bool have_dz_interface = false;
    double *acc_precip = nullptr;             // rain [0, nx*ny), snow [nx*ny, 2*nx*ny)
    int *mp_stop = nullptr;
    bool mp_ran = false;
    std::vector<DevBuf> qn, q1s;               // fused path: next state and pass-1 result per species
    bool fused_ready = false;
    bool std_ready = false;      // fused standard-scheme buffers and kernel attributes
    bool std_staged_ready = false;
    DevBuf fx, fy, fz, ufx, ufy, ufz, dq, sin_, sout, temp;  // STD scratch
    // 0 = fused kernels (MPDATA order 2, every standard-scheme setting), 1 = staged kernels,
    // 2 = single-pass MPDATA kernel (exact), 3 = single-pass MPDATA kernel (fast arithmetic)
    int path = 0;
    // single-pass kernel: TMA descriptors by device address (host cache),
    // two device tables of descriptors (the species buffers alternate between
    // two allocations, so two tables cover every step), timeout flag
    std::unordered_map<const float *, CUtensorMap> tmaps;
    CUtensorMap *map_dev[2] = {nullptr, nullptr};
    std::vector<const float *> map_tag[2];
    int map_next = 0;
    int *op_err = nullptr;
    bool op_ready = false;
    int mp_shape = 1;  // tile shape of the fused correction kernel (icar::mp_shape_ty)
    int sp_group = 0;  // species per thread of the fused upwind pass (0 = all)
    // diagnostics: launch counter and optional event timing of the species kernels
    int64_t launches = 0;
    int64_t timed_launches = 0;
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> corr_events;  // the fused correction kernel alone
    icar_adv_batch *batch = nullptr;  // batch this domain is a member of, if any
    std::string err;
};

namespace {

int fail(icar_adv_t *h, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h)
        h->err = buf;
    else
        g_create_error = buf;
    return code;
}

#define CUDA_TRY(h, call)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            return fail((h), e_ == cudaErrorMemoryAllocation ? ICAR_ADV_OOM : ICAR_ADV_CUDA_ERROR, \
                        "%s failed: %s", #call, cudaGetErrorString(e_));                           \
        }                                                                                          \
    } while (0)

bool is_species_id(int id) { return (id >= 7 && id <= 29 && id != 8); }

int halo_for(const icar_adv_opts &o)
{
    // read_domain_shape, src/objects/domain_obj.f90:2979-2986, and
    // set_grid_dimensions, src/objects/grid_obj.f90:153-154.
    int adv_order = std::max(o.h_order, o.v_order);
    if (o.flux_corr == ICAR_FLUXCOR_MONO) adv_order += 2;
    if (o.advection == ICAR_ADV_MPDATA) adv_order = 4;
    return (adv_order + 1) / 2;  // ceiling(adv_order/2.0)
}

int validate(const icar_adv_desc *d, const icar_adv_opts *o, std::string &why)
{
    char b[256];
    if (!d || !o) { why = "desc/opts is NULL"; return ICAR_ADV_BAD_ARG; }
    if (d->nx < 3 || d->ny < 3 || d->nz < 3) {
        snprintf(b, sizeof b, "domain %dx%dx%d too small (each extent must be >= 3)", d->nx, d->ny, d->nz);
        why = b; return ICAR_ADV_BAD_ARG;
    }
    if ((int64_t)d->nx * d->ny * d->nz > (int64_t)1 << 31) { why = "domain larger than 2^31 cells"; return ICAR_ADV_BAD_ARG; }
    if (!(d->dx > 0.0f) || !std::isfinite(d->dx)) { why = "dx must be positive"; return ICAR_ADV_BAD_ARG; }
    if (d->n_species < 0 || d->n_species > ICAR_ADV_MAX_SPECIES) { why = "n_species out of range"; return ICAR_ADV_BAD_ARG; }
    for (int s = 0; s < d->n_species; s++) {
        if (!is_species_id(d->species[s])) {
            snprintf(b, sizeof b, "species[%d]=%d is not an advectable kVARS id", s, d->species[s]);
            why = b; return ICAR_ADV_BAD_ARG;
        }
        for (int t = 0; t < s; t++)
            if (d->species[t] == d->species[s]) { why = "duplicate species id"; return ICAR_ADV_BAD_ARG; }
    }
    if (o->advection != ICAR_ADV_STD && o->advection != ICAR_ADV_MPDATA) { why = "advection must be 1 (STD) or 2 (MPDATA)"; return ICAR_ADV_BAD_ARG; }
    if (o->advection == ICAR_ADV_MPDATA && (o->mpdata_order < 1 || o->mpdata_order > 8)) { why = "mpdata_order must be 1..8"; return ICAR_ADV_BAD_ARG; }
    if (o->advection == ICAR_ADV_STD) {
        auto ok = [](int v) { return v == 1 || v == 3 || v == 5; };
        if (!ok(o->h_order) || !ok(o->v_order)) { why = "h_order and v_order must be 1, 3 or 5"; return ICAR_ADV_BAD_ARG; }
        if (o->flux_corr != 0 && o->flux_corr != 1) { why = "flux_corr must be 0 or 1"; return ICAR_ADV_BAD_ARG; }
        int hs = halo_for(*o);
        int need = 2 * hs + 1;
        if (d->nx < need || d->ny < need) { why = "domain smaller than twice the halo"; return ICAR_ADV_BAD_ARG; }
        int reach = o->h_order == 5 ? 3 : (o->h_order == 3 ? 2 : 1);
        if (o->flux_corr) reach += 1;
        if (reach > hs) { why = "stencil reaches past the halo"; return ICAR_ADV_BAD_ARG; }
    }
    return ICAR_ADV_OK;
}

void geometry(const icar_adv_desc &d, Geo &g, size_t &n_cell, size_t &n_u, size_t &n_v, size_t &n_zf)
{
    g.nx = d.nx; g.ny = d.ny; g.nz = d.nz;
    g.P = ((d.nx + 1) + 3) / 4 * 4;
    n_cell = (size_t)g.P * g.nz * g.ny;
    n_u = n_cell;
    n_v = (size_t)g.P * g.nz * (g.ny + 1);
    n_zf = (size_t)g.P * (g.nz + 1) * g.ny;
}

// Device bytes a handle allocates (create + the lazily allocated scratch).
int64_t footprint_bytes(const icar_adv_desc &d, const icar_adv_opts &o)
{
    Geo g; size_t nc, nu, nv, nzf;
    geometry(d, g, nc, nu, nv, nzf);
    int64_t f = 4;
    int64_t total = 0;
    total += f * (int64_t)(nu + nv + nc + nc * 2 + nu + nv + nc * 2);  // u v w rho jac ju jv jw dz
    total += f * (int64_t)nc * (d.n_species + 1);                      // species + spare
    total += f * (int64_t)(nu + nv + nc);                              // Um Vm Wm
    if (o.advection == ICAR_ADV_MPDATA && !o.rk3 && icar::fused_eligible(o.mpdata_order, o.mpdata_fct))
        total += f * (int64_t)nc * (2 * d.n_species + 3);              // fused: next + pass-1 per species, G, DJR, W'
    else if (o.advection == ICAR_ADV_MPDATA)
        total += f * (int64_t)(nc + 2 * (nu + nv + nc));               // staged scratch
    else
        total += f * (int64_t)nc * (2 * d.n_species + 2);              // fused: two stage results per species, G, DJR
    total += f * (int64_t)d.nx * d.ny + 4 * (int64_t)d.nx * d.ny;
    return total;
}

// Device memory of the handles comes from one stream-ordered memory pool
// per device that keeps freed memory for reuse (its release threshold is
// never reached).  Creating and destroying a handle then neither maps nor
// unmaps device memory, and destroying one does not wait for the device
// (cudaFree waits for every launch on the device): a request server that
// admits and retires many domains a second while its batched steps run
// depends on both.  Allocations are ordered on the handle's stream; the
// frees are ordered on it too, after all the work queued there.
constexpr int POOL_MAX_DEVICES = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pool[POOL_MAX_DEVICES] = {};

cudaError_t pool_of(int dev, cudaMemPool_t *out)
{
    if (dev < 0 || dev >= POOL_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pool[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        g_pool[dev] = p;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

// bytes of device memory for handle h, ordered on its stream
cudaError_t dev_alloc(icar_adv_t *h, void **p, size_t bytes)
{
    cudaMemPool_t pool;
    cudaError_t e = pool_of(h->desc.device, &pool);
    if (e != cudaSuccess) return e;
    e = cudaMallocFromPoolAsync(p, bytes, pool, h->stream);
    if (e != cudaSuccess) *p = nullptr;
    return e;
}

void dev_free(void *p, cudaStream_t st)
{
    if (p) cudaFreeAsync(p, st);
}

int alloc(icar_adv_t *h, DevBuf &b, size_t n)
{
    if (b.p) return ICAR_ADV_OK;
    cudaError_t e = dev_alloc(h, (void **)&b.p, n * sizeof(float));
    if (e != cudaSuccess) {
        b.p = nullptr;
        return fail(h, e == cudaErrorMemoryAllocation ? ICAR_ADV_OOM : ICAR_ADV_CUDA_ERROR,
                    "device allocation of %zu bytes failed: %s", n * sizeof(float), cudaGetErrorString(e));
    }
    b.n = n;
    h->bytes += n * sizeof(float);
    e = cudaMemsetAsync(b.p, 0, n * sizeof(float), h->stream);
    if (e != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaMemsetAsync failed: %s", cudaGetErrorString(e));
    return ICAR_ADV_OK;
}

void release(DevBuf &b, cudaStream_t st)
{
    dev_free(b.p, st);
    b.p = nullptr;
    b.n = 0;
}

// Host mirror of init_relax_filters (src/objects/domain_obj.f90:3285-3400).
void relax_filter(int nx, int ny, int hs, int north, int south, int east, int west, std::vector<float> &f)
{
    const float rs[7] = {0.9f, 0.75f, 0.6f, 0.5f, 0.4f, 0.25f, 0.1f};
    const float rs_r[7] = {0.1f, 0.25f, 0.4f, 0.5f, 0.6f, 0.75f, 0.9f};
    const int ims = 1, ime = nx, jms = 1, jme = ny;
    f.assign((size_t)nx * ny, 0.0f);
    bool corner = (west || east) && (north || south);
    int nr = std::min(7, std::min(ime - ims - hs, jme - jms - hs));
    auto set = [&](int i, int j, float val) {
        if (i >= 1 && i <= nx && j >= 1 && j <= ny) f[(size_t)(i - 1) + (size_t)nx * (j - 1)] = val;
    };
    if (!corner) {
        if (west) {
            for (int j = jms; j <= jme; j++) for (int i = ims; i <= ims + hs - 1; i++) set(i, j, 1.0f);
            for (int k = jms; k <= jme; k++) for (int m = 1; m <= nr; m++) set(ims + hs + m - 1, k, rs[m - 1]);
        } else if (east) {
            for (int j = jms; j <= jme; j++) for (int i = ime - hs + 1; i <= ime; i++) set(i, j, 1.0f);
            for (int k = jms; k <= jme; k++) for (int m = 1; m <= nr; m++) set(ime - hs - nr + m, k, rs_r[m - 1]);
        } else if (north) {
            for (int j = jme - hs - 1; j <= jme; j++) for (int i = ims; i <= ime; i++) set(i, j, 1.0f);
            for (int k = ims; k <= ime; k++) for (int m = 1; m <= nr; m++) set(k, jme - hs - nr + m, rs_r[m - 1]);
        } else if (south) {
            for (int j = jms; j <= jms + hs - 1; j++) for (int i = ims; i <= ime; i++) set(i, j, 1.0f);
            for (int k = ims; k <= ime; k++) for (int m = 1; m <= nr; m++) set(k, jms + hs + m - 1, rs[m - 1]);
        }
        return;
    }
    if (north && west) {
        for (int j = jms; j <= jme; j++) for (int i = ims; i <= ims + hs - 1; i++) set(i, j, 1.0f);
        for (int j = jme - hs - 1; j <= jme; j++) for (int i = ims; i <= ime; i++) set(i, j, 1.0f);
        for (int k = jms; k <= jme - hs; k++) for (int m = 1; m <= nr; m++) set(ims + hs + m - 1, k, rs[m - 1]);
        for (int k = ims + hs; k <= ime; k++) for (int m = 1; m <= nr; m++) set(k, jme - hs - nr + m, rs_r[m - 1]);
        for (int i = 1; i <= nr; i++) for (int k = 1; k <= nr; k++) set(ims + hs + i - 1, jme - hs - k + 1, rs[std::min(i, k) - 1]);
    } else if (north && east) {
        for (int j = jms; j <= jme; j++) for (int i = ime - hs + 1; i <= ime; i++) set(i, j, 1.0f);
        for (int j = jme - hs - 1; j <= jme; j++) for (int i = ims; i <= ime; i++) set(i, j, 1.0f);
        for (int k = jms; k <= jme - hs; k++) for (int m = 1; m <= nr; m++) set(ime - hs - nr + m, k, rs_r[m - 1]);
        for (int k = ims; k <= ime - hs; k++) for (int m = 1; m <= nr; m++) set(k, jme - hs - nr + m, rs_r[m - 1]);
        for (int i = 1; i <= nr; i++) for (int k = 1; k <= nr; k++) set(ime - hs - i + 1, jme - hs - k + 1, rs[std::min(i, k) - 1]);
    } else if (south && west) {
        for (int j = jms; j <= jme; j++) for (int i = ims; i <= ims + hs - 1; i++) set(i, j, 1.0f);
        for (int j = jms; j <= jms + hs - 1; j++) for (int i = ims; i <= ime; i++) set(i, j, 1.0f);
        for (int k = jms + hs; k <= jme; k++) for (int m = 1; m <= nr; m++) set(ims + hs + m - 1, k, rs[m - 1]);
        for (int k = ims + hs; k <= ime; k++) for (int m = 1; m <= nr; m++) set(k, jms + hs + m - 1, rs[m - 1]);
        for (int i = 1; i <= nr; i++) for (int k = 1; k <= nr; k++) set(ims + hs + i - 1, jms + hs + k - 1, rs[std::min(i, k) - 1]);
    } else if (south && east) {
        for (int j = jms; j <= jme; j++) for (int i = ime - hs + 1; i <= ime; i++) set(i, j, 1.0f);
        for (int j = jms; j <= jms + hs - 1; j++) for (int i = ims; i <= ime; i++) set(i, j, 1.0f);
        for (int k = jms + hs; k <= jme; k++) for (int m = 1; m <= nr; m++) set(ime - hs - nr + m, k, rs_r[m - 1]);
        for (int k = ims; k <= ime - hs; k++) for (int m = 1; m <= nr; m++) set(k, jms + hs + m - 1, rs[m - 1]);
        for (int i = 1; i <= nr; i++) for (int k = 1; k <= nr; k++) set(ime - hs - i + 1, jms + hs + k - 1, rs[std::min(i, k) - 1]);
    }
}

int upload_filter(icar_adv_t *h)
{
    std::vector<int> zone;
    for (int j = 0; j < h->g.ny; j++)
        for (int i = 0; i < h->g.nx; i++)
            if (h->filter_host[(size_t)i + (size_t)h->g.nx * j] != 0.0f) zone.push_back(i + h->g.nx * j);
    if (h->zone_dev) {
        dev_free(h->zone_dev, h->stream);
        h->zone_dev = nullptr;
    }
    h->nzone = (int)zone.size();
    if (!h->filter_dev) {
        CUDA_TRY(h, dev_alloc(h, (void **)&h->filter_dev, sizeof(float) * h->filter_host.size()));
        h->bytes += sizeof(float) * h->filter_host.size();
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->filter_dev, h->filter_host.data(), sizeof(float) * h->filter_host.size(),
                                cudaMemcpyHostToDevice, h->stream));
    if (h->nzone > 0) {
        CUDA_TRY(h, dev_alloc(h, (void **)&h->zone_dev, sizeof(int) * zone.size()));
        CUDA_TRY(h, cudaMemcpyAsync(h->zone_dev, zone.data(), sizeof(int) * zone.size(), cudaMemcpyHostToDevice,
                                    h->stream));
    }
    // the host vectors are the copies' sources
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    return ICAR_ADV_OK;
}

// A member's forcing buffers changed: its batch must rebuild tables and graphs.
void batch_fields_changed(icar_adv_batch *b);

// Resolve a field id to its device buffer, extents and presence flag.
struct FieldRef {
    DevBuf *buf = nullptr;
    int ex = 0, ey = 0;  // x extent (nx or nx+1) and y extent (ny or ny+1)
    int ez = 0;
    bool *flag = nullptr;
    int species = -1;
    bool is_forcing = false, is_dqdt = false, is_filter = false;
};

int species_slot(const icar_adv_t *h, int id)
{
    for (int s = 0; s < h->desc.n_species; s++)
        if (h->desc.species[s] == id) return s;
    return -1;
}

int resolve(icar_adv_t *h, int field, FieldRef &r)
{
    const int nx = h->g.nx, ny = h->g.ny, nz = h->g.nz;
    r.ez = nz;
    switch (field) {
    case ICAR_F_U: r = {&h->u, nx + 1, ny, nz, &h->have_u}; return ICAR_ADV_OK;
    case ICAR_F_V: r = {&h->v, nx, ny + 1, nz, &h->have_v}; return ICAR_ADV_OK;
    case ICAR_F_W: r = {&h->w, nx, ny, nz, &h->have_w}; return ICAR_ADV_OK;
    case ICAR_F_DENSITY: r = {&h->rho, nx, ny, nz, &h->have_rho}; return ICAR_ADV_OK;
    case ICAR_F_JACOBIAN: r = {&h->jac, nx, ny, nz, &h->have_jac}; return ICAR_ADV_OK;
    case ICAR_F_JACOBIAN_U: r = {&h->jac_u, nx + 1, ny, nz, &h->have_jac_u}; return ICAR_ADV_OK;
    case ICAR_F_JACOBIAN_V: r = {&h->jac_v, nx, ny + 1, nz, &h->have_jac_v}; return ICAR_ADV_OK;
    case ICAR_F_JACOBIAN_W: r = {&h->jac_w, nx, ny, nz, &h->have_jac_w}; return ICAR_ADV_OK;
    case ICAR_F_ADVECTION_DZ: r = {&h->dz, nx, ny, nz, &h->have_dz}; return ICAR_ADV_OK;
    case ICAR_F_RELAX_FILTER: r = FieldRef{}; r.ex = nx; r.ey = ny; r.ez = 1; r.is_filter = true; return ICAR_ADV_OK;
    case ICAR_F_DZ_INTERFACE: {
        int e = alloc(h, h->dz_interface, h->n_cell);
        if (e) return e;
        r = {&h->dz_interface, nx, ny, nz, &h->have_dz_interface};
        return ICAR_ADV_OK;
    }
    case ICAR_F_PRESSURE: case ICAR_F_EXNER: case ICAR_F_DZ_MASS: {
        DevBuf *b = field == ICAR_F_PRESSURE ? &h->pressure : field == ICAR_F_EXNER ? &h->exner : &h->dz_mass;
        bool *f = field == ICAR_F_PRESSURE ? &h->have_pressure : field == ICAR_F_EXNER ? &h->have_exner : &h->have_dz_mass;
        int e = alloc(h, *b, h->n_cell);
        if (e) return e;
        r = {b, nx, ny, nz, f};
        return ICAR_ADV_OK;
    }
    default: break;
    }
    int base = field;
    bool fo = false, dq = false;
    if (field >= ICAR_F_DQDT_BASE) { base = field - ICAR_F_DQDT_BASE; dq = true; }
    else if (field >= ICAR_F_FORCING_BASE) { base = field - ICAR_F_FORCING_BASE; fo = true; }
    int s = species_slot(h, base);
    if (s < 0) return fail(h, ICAR_ADV_BAD_ARG, "field id %d is not a field of this domain", field);
    r = FieldRef{};
    r.ex = nx; r.ey = ny; r.ez = nz; r.species = s; r.is_forcing = fo; r.is_dqdt = dq;
    if (fo) { int e = alloc(h, h->forcing[s], h->n_cell); if (e) return e; r.buf = &h->forcing[s]; }
    else if (dq) { int e = alloc(h, h->dqdt[s], h->n_cell); if (e) return e; r.buf = &h->dqdt[s]; }
    else r.buf = &h->q[s];
    if ((fo || dq) && h->batch) batch_fields_changed(h->batch);
    return ICAR_ADV_OK;
}

int copy_field(icar_adv_t *h, int field, float *host, const int64_t *strides, bool to_device, bool wait = true)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (!host) return fail(h, ICAR_ADV_BAD_ARG, "host pointer is NULL");
    FieldRef r;
    int e = resolve(h, field, r);
    if (e) return e;
    const int ex = r.ex, ey = r.ey, ez = r.ez;
    int64_t sx = 1, sz = ex, sy = (int64_t)ex * ez;
    if (strides) { sx = strides[0]; sz = strides[1]; sy = strides[2]; }
    if (r.is_filter) {
        if (to_device) {
            for (int j = 0; j < ey; j++)
                for (int i = 0; i < ex; i++) h->filter_host[(size_t)i + (size_t)ex * j] = host[i * sx + j * sy];
            return upload_filter(h);
        }
        for (int j = 0; j < ey; j++)
            for (int i = 0; i < ex; i++) host[i * sx + j * sy] = h->filter_host[(size_t)i + (size_t)ex * j];
        return ICAR_ADV_OK;
    }
    if (h->opts.debug && to_device) {
        for (int j = 0; j < ey; j++)
            for (int k = 0; k < ez; k++)
                for (int i = 0; i < ex; i++)
                    if (!std::isfinite(host[i * sx + k * sz + j * sy]))
                        return fail(h, ICAR_ADV_NAN_INPUT, "field %d has a non-finite value at (%d,%d,%d)", field, i + 1, k + 1, j + 1);
    }
    const size_t P = (size_t)h->g.P;
    if (sx == 1) {
        // rows of ex contiguous floats; rows of (k,j) are at k*sz + j*sy
        if (sy == sz * ez) {
            cudaError_t ce;
            if (to_device)
                ce = cudaMemcpy2DAsync(r.buf->p, P * 4, host, (size_t)sz * 4, (size_t)ex * 4, (size_t)ez * ey,
                                       cudaMemcpyHostToDevice, h->stream);
            else
                ce = cudaMemcpy2DAsync(host, (size_t)sz * 4, r.buf->p, P * 4, (size_t)ex * 4, (size_t)ez * ey,
                                       cudaMemcpyDeviceToHost, h->stream);
            if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaMemcpy2DAsync: %s", cudaGetErrorString(ce));
        } else {
            for (int j = 0; j < ey; j++) {
                cudaError_t ce;
                if (to_device)
                    ce = cudaMemcpy2DAsync(r.buf->p + P * ez * j, P * 4, host + sy * j, (size_t)sz * 4, (size_t)ex * 4,
                                           (size_t)ez, cudaMemcpyHostToDevice, h->stream);
                else
                    ce = cudaMemcpy2DAsync(host + sy * j, (size_t)sz * 4, r.buf->p + P * ez * j, P * 4, (size_t)ex * 4,
                                           (size_t)ez, cudaMemcpyDeviceToHost, h->stream);
                if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaMemcpy2DAsync: %s", cudaGetErrorString(ce));
            }
        }
    } else {
        // general strides: pack through a host staging buffer
        std::vector<float> stage((size_t)ex * ez * ey);
        if (to_device) {
            for (int j = 0; j < ey; j++)
                for (int k = 0; k < ez; k++)
                    for (int i = 0; i < ex; i++)
                        stage[(size_t)i + (size_t)ex * (k + (size_t)ez * j)] = host[i * sx + k * sz + j * sy];
            CUDA_TRY(h, cudaMemcpy2DAsync(r.buf->p, P * 4, stage.data(), (size_t)ex * 4, (size_t)ex * 4,
                                          (size_t)ez * ey, cudaMemcpyHostToDevice, h->stream));
            CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        } else {
            CUDA_TRY(h, cudaMemcpy2DAsync(stage.data(), (size_t)ex * 4, r.buf->p, P * 4, (size_t)ex * 4,
                                          (size_t)ez * ey, cudaMemcpyDeviceToHost, h->stream));
            CUDA_TRY(h, cudaStreamSynchronize(h->stream));
            for (int j = 0; j < ey; j++)
                for (int k = 0; k < ez; k++)
                    for (int i = 0; i < ex; i++)
                        host[i * sx + k * sz + j * sy] = stage[(size_t)i + (size_t)ex * (k + (size_t)ez * j)];
        }
    }
    if (to_device) {
        if (r.flag) *r.flag = true;
        if (r.species >= 0 && !r.is_forcing && !r.is_dqdt) h->have_q[r.species] = true;
    } else if (wait) {
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    }
    return ICAR_ADV_OK;
}

inline unsigned blocks_for(size_t n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

// After a sync: report (once) a column where mp_simple reached the
// reference's stop condition.
int check_mp_stop(icar_adv_t *h)
{
    if (!h->mp_ran || !h->mp_stop) return ICAR_ADV_OK;
    int flag = 0;
    cudaError_t e = cudaMemcpy(&flag, h->mp_stop, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "reading the mp stop flag: %s", cudaGetErrorString(e));
    h->mp_ran = false;
    if (!flag) return ICAR_ADV_OK;
    cudaMemset(h->mp_stop, 0, sizeof(int));
    return fail(h, ICAR_ADV_PHYSICS_STOP,
                "mp_simple: phase_change left a hydrometeor in [-1e-30, 0), where the reference stops");
}

int check_launch(icar_adv_t *h, const char *what, int n = 1)
{
    h->launches += n;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "launch of %s failed: %s", what, cudaGetErrorString(e));
    return ICAR_ADV_OK;
}

int ensure_ready(icar_adv_t *h)
{
    const char *missing = nullptr;
    if (!h->have_u) missing = "u";
    else if (!h->have_v) missing = "v";
    else if (!h->have_w) missing = "w";
    else if (!h->have_jac) missing = "jacobian";
    else if (!h->have_jac_u) missing = "jacobian_u";
    else if (!h->have_jac_v) missing = "jacobian_v";
    else if (!h->have_jac_w) missing = "jacobian_w";
    else if (!h->have_dz) missing = "advection_dz";
    else if (!h->have_rho && (h->opts.advection == ICAR_ADV_MPDATA || h->opts.advect_density)) missing = "density";
    if (missing) return fail(h, ICAR_ADV_NOT_READY, "field %s was never set", missing);
    for (int s = 0; s < h->desc.n_species; s++)
        if (!h->have_q[s]) return fail(h, ICAR_ADV_NOT_READY, "species %d was never set", h->desc.species[s]);
    return ICAR_ADV_OK;
}

// Courant fluxes for the step (mpdata_compute_wind or adv_std_compute_wind).
int compute_wind(icar_adv_t *h, float dt)
{
    const Geo &g = h->g;
    size_t n = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
    const float *rho = h->have_rho ? h->rho.p : h->jac.p;  // only read when advect_density
    if (h->opts.advection == ICAR_ADV_MPDATA)
        icar::k_mpdata_wind<<<blocks_for(n, 256), 256, 0, h->stream>>>(
            g, h->desc.dx, dt, h->opts.advect_density, h->u.p, h->v.p, h->w.p, rho, h->jac_u.p, h->jac_v.p,
            h->jac_w.p, h->Um.p, h->Vm.p, h->Wm.p);
    else
        icar::k_std_wind<<<blocks_for(n, 256), 256, 0, h->stream>>>(
            g, h->desc.dx, dt, h->opts.advect_density, h->u.p, h->v.p, h->w.p, rho, h->jac_u.p, h->jac_v.p,
            h->jac_w.p, h->dz.p, h->Um.p, h->Vm.p, h->Wm.p);
    return check_launch(h, "compute_wind", 1);
}

// MPDATA with the staged kernels (any mpdata_order, FCT on or off).
int mpdata_staged(icar_adv_t *h, int s)
{
    const Geo &g = h->g;
    {
        const size_t nc = h->n_cell, nu = h->n_u, nv = h->n_v;
        int e;
        if ((e = alloc(h, h->q1, nc)) || (e = alloc(h, h->u2, nu)) || (e = alloc(h, h->v2, nv)) ||
            (e = alloc(h, h->w2, nc)) || (e = alloc(h, h->u2l, nu)) || (e = alloc(h, h->v2l, nv)) ||
            (e = alloc(h, h->w2l, nc)))
            return e;
    }
    float *q = h->q[s].p;
    const size_t nc = (size_t)g.nx * g.nz * g.ny;
    const size_t nf = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
    const int order = h->opts.mpdata_order;
    for (int iord = 1; iord <= order; iord++) {
        if (iord == 1) {
            icar::k_upwind<<<blocks_for(nc, 256), 256, 0, h->stream>>>(g, q, h->Um.p, h->Vm.p, h->Wm.p, h->rho.p,
                                                                       h->jac.p, h->dz.p, h->q1.p);
        } else {
            icar::k_pseudo<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, h->q1.p, h->Um.p, h->Vm.p, h->Wm.p,
                                                                       h->rho.p, h->jac.p, h->dz.p, h->u2.p,
                                                                       h->v2.p, h->w2.p);
            const float *uu = h->u2.p, *vv = h->v2.p, *ww = h->w2.p;
            if (h->opts.mpdata_fct) {
                icar::k_fct<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, q, h->q1.p, h->u2.p, h->v2.p, h->w2.p,
                                                                        h->u2l.p, h->v2l.p, h->w2l.p);
                uu = h->u2l.p; vv = h->v2l.p; ww = h->w2l.p;
            }
            icar::k_upwind<<<blocks_for(nc, 256), 256, 0, h->stream>>>(g, h->q1.p, uu, vv, ww, h->rho.p, h->jac.p,
                                                                       h->dz.p, q);
        }
        if (iord != order) {
            if (iord > 1)
                if (cudaMemcpyAsync(h->q1.p, q, h->n_cell * 4, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
                    return fail(h, ICAR_ADV_CUDA_ERROR, "copy q -> q2 failed");
        } else if (iord == 1) {
            if (cudaMemcpyAsync(q, h->q1.p, h->n_cell * 4, cudaMemcpyDeviceToDevice, h->stream) != cudaSuccess)
                return fail(h, ICAR_ADV_CUDA_ERROR, "copy q2 -> q failed");
        }
    }
    return check_launch(h, "mpdata staged kernels", 1 + (order - 1) * (h->opts.mpdata_fct ? 3 : 2));
}

// One adv_std_advect3d call: fluxes from qf scaled by t_factor, optional WRF
// correction against qold, update written to qout (may alias qold).
// Scratch of the staged standard scheme (flux arrays, RK3 temporary, WRF
// work arrays), allocated on first use.
int ensure_std_staged(icar_adv_t *h)
{
    if (h->std_staged_ready) return ICAR_ADV_OK;
    const size_t nc = h->n_cell, nu = h->n_u, nv = h->n_v;
    int e;
    if ((e = alloc(h, h->fx, nu)) || (e = alloc(h, h->fy, nv)) || (e = alloc(h, h->fz, h->n_zf)) ||
        (e = alloc(h, h->temp, nc)))
        return e;
    if (h->opts.flux_corr == 1)
        if ((e = alloc(h, h->ufx, nu)) || (e = alloc(h, h->ufy, nv)) || (e = alloc(h, h->ufz, h->n_zf)) ||
            (e = alloc(h, h->dq, nc)) || (e = alloc(h, h->sin_, nc)) || (e = alloc(h, h->sout, nc)))
            return e;
    h->std_staged_ready = true;
    return ICAR_ADV_OK;
}

// Callers run ensure_std_staged first (qout may be the scratch temp array).
int std_advect3d(icar_adv_t *h, const float *qf, const float *qold, float *qout, float t_factor, int flux_corr)
{
    const Geo &g = h->g;
    const int hs = h->hs;
    const int its = hs, ite = g.nx - 1 - hs, jts = hs, jte = g.ny - 1 - hs;
    int is = its, ie = ite, js = jts, je = jte;
    if (flux_corr == 1) { is--; ie++; js--; je++; }
    const size_t nf = (size_t)(g.nx + 1) * (g.nz + 1) * (g.ny + 1);
    const size_t nc = (size_t)g.nx * g.nz * g.ny;
    const float *rho = h->have_rho ? h->rho.p : h->jac.p;
    const int ad = h->opts.advect_density;
    icar::k_flux3<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, h->opts.h_order, h->opts.v_order, is, ie, js, je,
                                                              t_factor, qf, h->Um.p, h->Vm.p, h->Wm.p, h->fx.p,
                                                              h->fy.p, h->fz.p);
    if (flux_corr == 1) {
        icar::k_upflux<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, 0, is, ie, js, je, qold, h->Um.p, h->Vm.p,
                                                                   h->Wm.p, h->ufx.p, h->ufy.p, h->ufz.p);
        icar::k_upflux_predict<<<blocks_for(nc, 256), 256, 0, h->stream>>>(g, is, ie, js, je, qold, h->ufx.p,
                                                                           h->ufy.p, h->ufz.p, h->jac.p, rho, ad,
                                                                           h->dz.p, h->dq.p);
        icar::k_upflux<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, 1, is, ie, js, je, h->dq.p, h->Um.p, h->Vm.p,
                                                                   h->Wm.p, h->ufx.p, h->ufy.p, h->ufz.p);
        icar::k_wrf_merge<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, is, ie, js, je, h->fx.p, h->fy.p, h->fz.p,
                                                                      h->ufx.p, h->ufy.p, h->ufz.p);
        icar::k_wrf_cells<<<blocks_for(nc, 256), 256, 0, h->stream>>>(
            g, is, ie, js, je, qold, h->Um.p, h->Vm.p, h->Wm.p, h->fx.p, h->fy.p, h->fz.p, h->ufx.p, h->ufy.p,
            h->ufz.p, h->jac.p, rho, ad, h->dz.p, h->sin_.p, h->sout.p);
        icar::k_wrf_scale<<<blocks_for(nf, 256), 256, 0, h->stream>>>(g, its, ite, jts, jte, h->fx.p, h->fy.p,
                                                                      h->fz.p, h->ufx.p, h->ufy.p, h->ufz.p,
                                                                      h->sin_.p, h->sout.p);
    }
    icar::k_std_update<<<blocks_for(nc, 256), 256, 0, h->stream>>>(g, its, ite, jts, jte, qold, h->fx.p, h->fy.p,
                                                                   h->fz.p, h->jac.p, rho, ad, h->dz.p, qout);
    return check_launch(h, "std kernels", flux_corr == 1 ? 8 : 2);
}

// Fused MPDATA (order 2): prep -> pass 1 for all species -> fused
// pseudo-velocity/FCT/corrective pass for all species, then swap buffers.
int ensure_fused(icar_adv_t *h)
{
    const int S = h->desc.n_species;
    int e;
    if (!h->fused_ready) {
        h->qn.resize(S);
        h->q1s.resize(S);
        if ((e = alloc(h, h->Gc, h->n_cell)) || (e = alloc(h, h->DJR, h->n_cell)) || (e = alloc(h, h->Wp, h->n_cell)))
            return e;
        for (int s = 0; s < S; s++)
            if ((e = alloc(h, h->qn[s], h->n_cell)) || (e = alloc(h, h->q1s[s], h->n_cell))) return e;
        cudaError_t ce = icar::mp_corr_setup();
        if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaFuncSetAttribute: %s", cudaGetErrorString(ce));
        h->fused_ready = true;
    }
    return ICAR_ADV_OK;
}

// ---------------------------------------------------------------------------
// Single-pass MPDATA kernel (mpdata_onepass.cuh): per-step fields from
// k_mp_prep, then one launch for every species.  It needs no pass-1
// buffers; its inputs are read through TMA descriptors.
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 tma_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Descriptor of one pitched 3-D field (rows = ny or ny+1) for 64 x 1 x 32
// plane boxes; cached per device address.
int plane_map(icar_adv_t *h, const float *base, int rows, const CUtensorMap **out)
{
    auto it = h->tmaps.find(base);
    if (it != h->tmaps.end()) {
        *out = &it->second;
        return ICAR_ADV_OK;
    }
    auto enc = tma_encoder();
    if (!enc) return fail(h, ICAR_ADV_CUDA_ERROR, "cuTensorMapEncodeTiled is not available from the driver");
    const Geo &g = h->g;
    CUtensorMap m;
    cuuint64_t dims[3] = {(cuuint64_t)g.P, (cuuint64_t)g.nz, (cuuint64_t)rows};
    cuuint64_t strides[2] = {(cuuint64_t)g.P * sizeof(float), (cuuint64_t)g.P * g.nz * sizeof(float)};
    cuuint32_t box[3] = {(cuuint32_t)icar::op::PW, 1u, (cuuint32_t)icar::op::PH};
    cuuint32_t es[3] = {1u, 1u, 1u};
    CUresult r = enc(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(h, ICAR_ADV_CUDA_ERROR, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    auto ins = h->tmaps.emplace(base, m);
    *out = &ins.first->second;
    return ICAR_ADV_OK;
}

// The device table of descriptors for the current buffers: every species
// input in adv_vars order, then U_m, V_m, W_m/dz, J*rho.  Two tables are
// kept, tagged with the device addresses they describe; a table is rebuilt
// (encode + one copy on the handle's stream) only when neither matches.
int onepass_maps(icar_adv_t *h, const CUtensorMap **out)
{
    const int S = h->desc.n_species;
    std::vector<const float *> want;
    want.reserve(S + 4);
    for (int s = 0; s < S; s++) want.push_back(h->q[s].p);
    want.push_back(h->Um.p);
    want.push_back(h->Vm.p);
    want.push_back(h->Wp.p);
    want.push_back(h->Gc.p);
    for (int t = 0; t < 2; t++)
        if (h->map_dev[t] && h->map_tag[t] == want) {
            *out = h->map_dev[t];
            return ICAR_ADV_OK;
        }
    const int t = h->map_next;
    h->map_next ^= 1;
    if (!h->map_dev[t]) CUDA_TRY(h, dev_alloc(h, (void **)&h->map_dev[t], (size_t)(S + 4) * sizeof(CUtensorMap)));
    std::vector<CUtensorMap> host(S + 4);
    int e;
    const CUtensorMap *m;
    for (int s = 0; s < S + 4; s++) {
        const int rows = s == S + 1 ? h->g.ny + 1 : h->g.ny;  // V_m has ny+1 rows
        if ((e = plane_map(h, want[s], rows, &m))) return e;
        host[s] = *m;
    }
    // ordered on the stream after any kernel still reading the old table
    CUDA_TRY(h, cudaMemcpyAsync(h->map_dev[t], host.data(), host.size() * sizeof(CUtensorMap),
                                cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->map_tag[t] = want;
    *out = h->map_dev[t];
    return ICAR_ADV_OK;
}

template <bool EXACT>
cudaError_t onepass_attr()
{
    cudaError_t e = cudaFuncSetAttribute(icar::k_mpdata_onepass<EXACT, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)icar::op::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(icar::k_mpdata_onepass<EXACT, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)icar::op::SMEM);
    return e;
}

int ensure_onepass(icar_adv_t *h)
{
    const int S = h->desc.n_species;
    int e;
    if (!h->op_ready) {
        h->qn.resize(S);
        if ((e = alloc(h, h->Gc, h->n_cell)) || (e = alloc(h, h->DJR, h->n_cell)) || (e = alloc(h, h->Wp, h->n_cell)))
            return e;
        for (int s = 0; s < S; s++)
            if ((e = alloc(h, h->qn[s], h->n_cell))) return e;
        if (!h->op_err) {
            CUDA_TRY(h, dev_alloc(h, (void **)&h->op_err, sizeof(int)));
            CUDA_TRY(h, cudaMemsetAsync(h->op_err, 0, sizeof(int), h->stream));
        }
        cudaError_t ce = onepass_attr<true>();
        if (ce == cudaSuccess) ce = onepass_attr<false>();
        if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaFuncSetAttribute: %s", cudaGetErrorString(ce));
        h->op_ready = true;
    }
    return ICAR_ADV_OK;
}

int onepass_tiles_x(const Geo &g) { return icar::op::tiles_x(g.nx); }
int onepass_tiles_y(const Geo &g) { return (g.ny + icar::op::TY - 1) / icar::op::TY; }

// The corrective pass and the donor-cell pass for species [s0, s1) in one
// launch; results in qn.
int mpdata_onepass_group(icar_adv_t *h, int s0, int s1)
{
    const Geo &g = h->g;
    const int S = s1 - s0;
    if (S <= 0) return ICAR_ADV_OK;
    icar::OnePassParams prm{};
    int e;
    const CUtensorMap *table = nullptr;
    if ((e = onepass_maps(h, &table))) return e;
    prm.q0maps = table + s0;
    prm.fmaps = table + h->desc.n_species;
    for (int s = 0; s < S; s++) prm.out[s] = h->qn[s0 + s].p;
    prm.Wm = h->Wm.p;
    prm.DJR = h->DJR.p;
    prm.dz = h->dz.p;
    prm.err = h->op_err;
    prm.g = g;
    prm.nspecies = S;
    prm.tiles_x = onepass_tiles_x(g);
    const unsigned grid = (unsigned)(onepass_tiles_x(g) * onepass_tiles_y(g) * S);
    const bool exact = h->path != 3, fct = h->opts.mpdata_fct != 0;
    cudaEvent_t c0 = nullptr, c1 = nullptr;
    if (h->profiling) {
        cudaEventCreate(&c0);
        cudaEventCreate(&c1);
        cudaEventRecord(c0, h->stream);
    }
    if (exact && fct) icar::k_mpdata_onepass<true, true><<<grid, icar::op::NT, icar::op::SMEM, h->stream>>>(prm);
    else if (exact) icar::k_mpdata_onepass<true, false><<<grid, icar::op::NT, icar::op::SMEM, h->stream>>>(prm);
    else if (fct) icar::k_mpdata_onepass<false, true><<<grid, icar::op::NT, icar::op::SMEM, h->stream>>>(prm);
    else icar::k_mpdata_onepass<false, false><<<grid, icar::op::NT, icar::op::SMEM, h->stream>>>(prm);
    if (h->profiling) {
        cudaEventRecord(c1, h->stream);
        h->corr_events.emplace_back(c0, c1);
    }
    return check_launch(h, "single-pass MPDATA kernel", 1);
}

// Species-independent part of the fused MPDATA step (Courant fluxes, G,
// DJR, W').
int mpdata_prep(icar_adv_t *h, float dt)
{
    const Geo &g = h->g;
    int e = h->path >= 2 ? ensure_onepass(h) : ensure_fused(h);
    if (e) return e;
    const size_t nf = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
    icar::k_mp_prep<<<blocks_for(nf, 256), 256, 0, h->stream>>>(
        g, h->desc.dx, dt, h->opts.advect_density, h->u.p, h->v.p, h->w.p, h->rho.p, h->jac.p, h->jac_u.p,
        h->jac_v.p, h->jac_w.p, h->dz.p, h->Um.p, h->Vm.p, h->Wm.p, h->Gc.p, h->DJR.p, h->Wp.p);
    if (h->opts.debug &&
        icar::check_courant(h->stream, h->g, h->Um.p, h->Vm.p, h->Wm.p, h->dz.p, h->jac.p, h->rho.p, 1))
        return fail(h, ICAR_ADV_CFL_VIOLATION, "a Courant number >= 1 was found (debug check)");
    return check_launch(h, "fused MPDATA prep", 1);
}

// Donor-cell pass and fused correction for species [s0, s1); results in qn.
int mpdata_group(icar_adv_t *h, int s0, int s1)
{
    const Geo &g = h->g;
    const int S = s1 - s0;
    if (S <= 0) return ICAR_ADV_OK;
    icar::SpeciesPtrs sp{};
    for (int s = 0; s < S; s++) {
        sp.q0[s] = h->q[s0 + s].p;
        sp.q1[s] = h->q1s[s0 + s].p;
        sp.out[s] = h->qn[s0 + s].p;
    }
    const int sg = std::min(icar::upwind_group(S, h->sp_group), icar::upf::SGMAX);
    const dim3 gu((unsigned)((g.nx + icar::upf::BX - 1) / icar::upf::BX),
                  (unsigned)((g.ny + icar::upf::BY - 1) / icar::upf::BY), (unsigned)((S + sg - 1) / sg));
    icar::k_mp_upwind_cols<<<gu, icar::upf::NT, icar::upf::SMEM, h->stream>>>(g, sp, S, sg, h->Um.p, h->Vm.p, h->Wm.p,
                                                                            h->Gc.p, h->DJR.p);
    cudaEvent_t c0 = nullptr, c1 = nullptr;
    if (h->profiling) {
        cudaEventCreate(&c0);
        cudaEventCreate(&c1);
        cudaEventRecord(c0, h->stream);
    }
    icar::mp_corr_launch(h->stream, h->mp_shape, g, sp, S, h->opts.mpdata_fct, h->Um.p, h->Vm.p, h->Wp.p, h->Gc.p,
                         h->DJR.p, h->dz.p);
    if (h->profiling) {
        cudaEventRecord(c1, h->stream);
        h->corr_events.emplace_back(c0, c1);
    }
    return check_launch(h, "fused MPDATA kernels", 2);
}

int mpdata_fused_step(icar_adv_t *h, float dt)
{
    const int S = h->desc.n_species;
    int e = mpdata_prep(h, dt);
    if (e) return e;
    if ((e = h->path >= 2 ? mpdata_onepass_group(h, 0, S) : mpdata_group(h, 0, S))) return e;
    for (int s = 0; s < S; s++) std::swap(h->q[s], h->qn[s]);
    return ICAR_ADV_OK;
}

// Fused standard scheme: prep (Courant fluxes, G, DJR) then one launch per
// adv_std_advect3d call for all species (three with RK3), results in
// per-species buffers swapped into place.
int ensure_std_fused(icar_adv_t *h)
{
    const int S = h->desc.n_species;
    int e;
    if (!h->std_ready) {
        h->qn.resize(S);
        h->q1s.resize(S);
        if ((e = alloc(h, h->Gc, h->n_cell)) || (e = alloc(h, h->DJR, h->n_cell))) return e;
        for (int s = 0; s < S; s++)
            if ((e = alloc(h, h->qn[s], h->n_cell)) || (e = alloc(h, h->q1s[s], h->n_cell))) return e;
        cudaError_t ce = icar::std_fused_setup();
        if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaFuncSetAttribute: %s", cudaGetErrorString(ce));
        h->std_ready = true;
    }
    return ICAR_ADV_OK;
}

// Species-independent part of the fused standard scheme (Courant fluxes,
// G, DJR).
int std_prep(icar_adv_t *h, float dt)
{
    const Geo &g = h->g;
    int e = ensure_std_fused(h);
    if (e) return e;
    const size_t nf = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
    const float *rho = h->have_rho ? h->rho.p : h->jac.p;  // only read when advect_density
    icar::k_std_prep<<<blocks_for(nf, 256), 256, 0, h->stream>>>(
        g, h->desc.dx, dt, h->opts.advect_density, h->u.p, h->v.p, h->w.p, rho, h->jac.p, h->jac_u.p, h->jac_v.p,
        h->jac_w.p, h->dz.p, h->Um.p, h->Vm.p, h->Wm.p, h->Gc.p, h->DJR.p);
    if (h->opts.debug &&
        icar::check_courant(h->stream, h->g, h->Um.p, h->Vm.p, h->Wm.p, h->dz.p, h->jac.p, h->rho.p,
                            h->opts.advect_density))
        return fail(h, ICAR_ADV_CFL_VIOLATION, "a Courant number >= 1 was found (debug check)");
    return check_launch(h, "fused standard-scheme prep", 1);
}

// The adv_std_advect3d calls of one step for species [s0, s1); results in
// q1s with RK3, in qn otherwise.
int std_group(icar_adv_t *h, int s0, int s1)
{
    const Geo &g = h->g;
    const int S = s1 - s0;
    if (S <= 0) return ICAR_ADV_OK;
    const int ho = h->opts.h_order, vo = h->opts.v_order, hs = h->hs;
    const bool corr = h->opts.flux_corr == 1;
    auto stage = [&](std::vector<DevBuf> *qf, std::vector<DevBuf> *out, float tf, bool c) {
        icar::SpeciesPtrs sp{};
        for (int s = 0; s < S; s++) {
            sp.q0[s] = h->q[s0 + s].p;
            sp.q1[s] = (qf ? *qf : h->q)[s0 + s].p;
            sp.out[s] = (*out)[s0 + s].p;
        }
        return icar::std_fused_launch(h->stream, c, ho, vo, g, hs, tf, sp, S, h->Um.p, h->Vm.p, h->Wm.p, h->Gc.p,
                                      h->DJR.p);
    };
    cudaEvent_t c0 = nullptr, c1 = nullptr;
    if (h->profiling) {
        cudaEventCreate(&c0);
        cudaEventCreate(&c1);
        cudaEventRecord(c0, h->stream);
    }
    int bad = 0, nl = 0;
    if (h->opts.rk3) {
        // advection_driver.f90:100-110: q + 1/3, q + 1/2 from the first
        // result, then the full step (with the flux correction) from the second
        bad |= stage(nullptr, &h->q1s, 0.333f, false);
        bad |= stage(&h->q1s, &h->qn, 0.5f, false);
        bad |= stage(&h->qn, &h->q1s, 1.0f, corr);
        nl = 6;
    } else {
        bad |= stage(nullptr, &h->qn, 1.0f, corr);
        nl = 2;
    }
    if (h->profiling) {
        cudaEventRecord(c1, h->stream);
        h->corr_events.emplace_back(c0, c1);
    }
    if (bad) return fail(h, ICAR_ADV_BAD_ARG, "h_order and v_order must be 1, 3 or 5");
    return check_launch(h, "fused standard-scheme kernels", nl);
}

int std_fused_step(icar_adv_t *h, float dt)
{
    const int S = h->desc.n_species;
    int e = std_prep(h, dt);
    if (e) return e;
    if ((e = std_group(h, 0, S))) return e;
    for (int s = 0; s < S; s++) std::swap(h->q[s], h->opts.rk3 ? h->q1s[s] : h->qn[s]);
    return ICAR_ADV_OK;
}

int advect_impl(icar_adv_t *h, float dt)
{
    int e = ensure_ready(h);
    if (e) return e;
    if (!(dt >= 0.0f) || !std::isfinite(dt)) return fail(h, ICAR_ADV_BAD_ARG, "dt must be finite and >= 0");
    const bool mp = h->opts.advection == ICAR_ADV_MPDATA;
    const bool fused_mp = mp && !h->opts.rk3 && icar::fused_eligible(h->opts.mpdata_order, h->opts.mpdata_fct);
    if ((h->path == 0 && (fused_mp || !mp)) || (h->path >= 2 && (fused_mp || !mp))) {
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        int64_t before = h->launches;
        if (h->profiling) {
            cudaEventCreate(&ev0);
            cudaEventCreate(&ev1);
            cudaEventRecord(ev0, h->stream);
        }
        e = mp ? mpdata_fused_step(h, dt) : std_fused_step(h, dt);
        if (e) return e;
        if (h->profiling) {
            cudaEventRecord(ev1, h->stream);
            h->events.emplace_back(ev0, ev1);
            h->timed_launches += h->launches - before;
        }
        return ICAR_ADV_OK;
    }
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int64_t before = h->launches;
    if (h->profiling) {
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, h->stream);
    }
    e = compute_wind(h, dt);
    if (e) return e;
    if (!mp && (e = ensure_std_staged(h))) return e;
    if (h->opts.debug) {
        e = icar::check_courant(h->stream, h->g, h->Um.p, h->Vm.p, h->Wm.p, h->dz.p, h->jac.p, h->rho.p,
                                h->opts.advect_density || mp);
        if (e) return fail(h, ICAR_ADV_CFL_VIOLATION, "a Courant number >= 1 was found (debug check)");
    }
    for (int s = 0; s < h->desc.n_species; s++) {
        if (h->opts.rk3) {
            if (!mp) {
                float *q = h->q[s].p;
                if ((e = std_advect3d(h, q, q, h->temp.p, 0.333f, 0))) return e;
                if ((e = std_advect3d(h, h->temp.p, q, h->temp.p, 0.5f, 0))) return e;
                if ((e = std_advect3d(h, h->temp.p, q, q, 1.0f, h->opts.flux_corr))) return e;
            }
            // MPDATA with RK3 does nothing in the reference (advection_driver.f90:112-115)
        } else if (!mp) {
            float *q = h->q[s].p;
            if ((e = std_advect3d(h, q, q, q, 1.0f, h->opts.flux_corr))) return e;
        } else {
            if ((e = mpdata_staged(h, s))) return e;
        }
    }
    if (h->profiling) {
        cudaEventRecord(ev1, h->stream);
        h->events.emplace_back(ev0, ev1);
        h->timed_launches += h->launches - before;
    }
    return ICAR_ADV_OK;
}

}  // namespace

extern "C" {

int icar_adv_abi_version(void) { return ICAR_ADV_ABI_VERSION; }

int icar_adv_default_opts(icar_adv_opts *o)
{
    if (!o) return fail(nullptr, ICAR_ADV_BAD_ARG, "opts is NULL");
    memset(o, 0, sizeof(*o));
    o->advection = ICAR_ADV_MPDATA;
    o->mpdata_fct = 1;
    o->mpdata_order = 2;
    o->flux_corr = 0;
    o->h_order = 1;
    o->v_order = 1;
    return ICAR_ADV_OK;
}

int icar_adv_var_request(const icar_adv_opts *opts, int32_t *alloc_vars, int32_t *n_alloc, int32_t *advect_vars,
                         int32_t *n_advect)
{
    if (!opts || !n_alloc || !n_advect) return fail(nullptr, ICAR_ADV_BAD_ARG, "NULL argument");
    // Both schemes request through adv_std_var_request (advection_driver.f90:52-56).
    const int32_t alloc[5] = {ICAR_F_U, ICAR_F_V, ICAR_F_W, ICAR_F_DZ_INTERFACE, ICAR_F_QV};
    const int32_t adv[2] = {ICAR_F_QV, ICAR_F_THETA};
    if (*n_alloc < 5 || *n_advect < 2 || !alloc_vars || !advect_vars) {
        *n_alloc = 5;
        *n_advect = 2;
        return fail(nullptr, ICAR_ADV_BAD_ARG, "output arrays need room for 5 and 2 ids");
    }
    memcpy(alloc_vars, alloc, sizeof alloc);
    memcpy(advect_vars, adv, sizeof adv);
    *n_alloc = 5;
    *n_advect = 2;
    return ICAR_ADV_OK;
}

int icar_adv_halo_size(const icar_adv_opts *opts)
{
    if (!opts) return -1;
    return halo_for(*opts);
}

int icar_adv_footprint(const icar_adv_desc *desc, const icar_adv_opts *opts, int64_t *bytes)
{
    std::string why;
    int e = validate(desc, opts, why);
    if (e) return fail(nullptr, e, "%s", why.c_str());
    if (!bytes) return fail(nullptr, ICAR_ADV_BAD_ARG, "bytes is NULL");
    *bytes = footprint_bytes(*desc, *opts);
    return ICAR_ADV_OK;
}

int icar_adv_create(const icar_adv_desc *desc, const icar_adv_opts *opts, icar_adv_t **out)
{
    if (!out) return fail(nullptr, ICAR_ADV_BAD_ARG, "out is NULL");
    *out = nullptr;
    std::string why;
    int e = validate(desc, opts, why);
    if (e) return fail(nullptr, e, "%s", why.c_str());
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0)
        return fail(nullptr, ICAR_ADV_CUDA_ERROR, "no CUDA device available: %s", cudaGetErrorString(ce));
    if (desc->device < 0 || desc->device >= ndev) return fail(nullptr, ICAR_ADV_BAD_ARG, "device %d out of range", desc->device);
    ce = cudaSetDevice(desc->device);
    if (ce != cudaSuccess) return fail(nullptr, ICAR_ADV_CUDA_ERROR, "cudaSetDevice: %s", cudaGetErrorString(ce));

    icar_adv_t *h = new icar_adv_domain();
    h->desc = *desc;
    h->opts = *opts;
    h->hs = halo_for(*opts);
    geometry(*desc, h->g, h->n_cell, h->n_u, h->n_v, h->n_zf);
    ce = cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) {
        delete h;
        return fail(nullptr, ICAR_ADV_CUDA_ERROR, "cudaStreamCreate: %s", cudaGetErrorString(ce));
    }
    h->stream = h->own_stream;
    const int S = desc->n_species;
    h->q.resize(S);
    h->have_q.assign(S, false);
    h->forcing.resize(S);
    h->dqdt.resize(S);
    auto bail = [&](int code) {
        g_create_error = h->err;
        icar_adv_destroy(h);
        return code;
    };
    const size_t nc = h->n_cell, nu = h->n_u, nv = h->n_v;
    if ((e = alloc(h, h->u, nu)) || (e = alloc(h, h->v, nv)) || (e = alloc(h, h->w, nc)) ||
        (e = alloc(h, h->rho, nc)) || (e = alloc(h, h->jac, nc)) || (e = alloc(h, h->jac_u, nu)) ||
        (e = alloc(h, h->jac_v, nv)) || (e = alloc(h, h->jac_w, nc)) || (e = alloc(h, h->dz, nc)) ||
        (e = alloc(h, h->Um, nu)) || (e = alloc(h, h->Vm, nv)) || (e = alloc(h, h->Wm, nc)) ||
        (e = alloc(h, h->spare, nc)))
        return bail(e);
    for (int s = 0; s < S; s++)
        if ((e = alloc(h, h->q[s], nc))) return bail(e);
    // the scratch of either scheme is allocated on first use (ensure_fused,
    // ensure_std_fused, mpdata_staged, std_advect3d)
    relax_filter(desc->nx, desc->ny, h->hs, desc->north_boundary, desc->south_boundary, desc->east_boundary,
                 desc->west_boundary, h->filter_host);
    if ((e = upload_filter(h))) return bail(e);
    ce = cudaStreamSynchronize(h->stream);
    if (ce != cudaSuccess) {
        h->err = std::string("initialisation failed: ") + cudaGetErrorString(ce);
        return bail(ICAR_ADV_CUDA_ERROR);
    }
    *out = h;
    return ICAR_ADV_OK;
}

int icar_adv_batch_remove(icar_adv_batch_t *b, icar_adv_t *member);

int icar_adv_destroy(icar_adv_t *h)
{
    if (!h) return ICAR_ADV_OK;
    if (h->batch) icar_adv_batch_remove(h->batch, h);
    cudaSetDevice(h->desc.device);
    // copies through the caller's host buffers end before this returns
    if (h->io_in) cudaStreamSynchronize(h->io_in);
    if (h->io_out) cudaStreamSynchronize(h->io_out);
    // The device memory goes back to the pool in the order of the handle's
    // own stream, after all the work queued on the stream it runs on (a
    // former batch member's own stream already waits for the batch launches
    // queued before its removal), so nothing here waits for the device.  If
    // the handle ran on a caller's stream that is gone, the device is
    // synchronised instead.
    cudaStream_t st = h->own_stream;
    if (h->stream != h->own_stream) {
        cudaEvent_t ev = nullptr;
        bool ordered = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) == cudaSuccess &&
                       cudaEventRecord(ev, h->stream) == cudaSuccess &&
                       cudaStreamWaitEvent(st, ev, 0) == cudaSuccess;
        if (ev) cudaEventDestroy(ev);
        if (!ordered) {
            cudaGetLastError();
            cudaDeviceSynchronize();
        }
    }
    for (DevBuf *b : {&h->u, &h->v, &h->w, &h->rho, &h->jac, &h->jac_u, &h->jac_v, &h->jac_w, &h->dz, &h->Um,
                      &h->Vm, &h->Wm, &h->spare, &h->q1, &h->u2, &h->v2, &h->w2, &h->u2l, &h->v2l, &h->w2l, &h->fx,
                      &h->fy, &h->fz, &h->ufx, &h->ufy, &h->ufz, &h->dq, &h->sin_, &h->sout, &h->temp, &h->Gc,
                      &h->DJR, &h->Wp, &h->dtbuf, &h->pressure, &h->exner, &h->dz_mass, &h->dz_interface})
        release(*b, st);
    dev_free(h->acc_precip, st);
    dev_free(h->mp_stop, st);
    dev_free(h->op_err, st);
    for (auto *m : h->map_dev) dev_free(m, st);
    for (auto &b : h->q) release(b, st);
    for (auto &b : h->qn) release(b, st);
    for (auto &b : h->q1s) release(b, st);
    for (auto &b : h->forcing) release(b, st);
    for (auto &b : h->dqdt) release(b, st);
    dev_free(h->filter_dev, st);
    dev_free(h->zone_dev, st);
    for (auto *v : {&h->events, &h->corr_events})
        for (auto &p : *v) {
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
    for (cudaEvent_t ev : h->io_events) cudaEventDestroy(ev);
    if (h->io_in) cudaStreamDestroy(h->io_in);
    if (h->io_out) cudaStreamDestroy(h->io_out);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);   // its queued frees still run
    delete h;
    return ICAR_ADV_OK;
}

int icar_adv_set_field(icar_adv_t *h, int32_t field, const float *host, const int64_t *strides)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    return copy_field(h, field, const_cast<float *>(host), strides, true);
}

int icar_adv_get_field(icar_adv_t *h, int32_t field, float *host, const int64_t *strides)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    return copy_field(h, field, host, strides, false);
}

int icar_adv_restart_vars(const icar_adv_opts *opts, int32_t *vars, int32_t *n)
{
    // adv_std_var_request, src/physics/advect.f90:95-107: the same set for
    // both schemes (advection_driver.f90:46-56)
    (void)opts;
    if (!n) return fail(nullptr, ICAR_ADV_BAD_ARG, "n is NULL");
    const int32_t set[5] = {ICAR_F_U, ICAR_F_V, ICAR_F_W, ICAR_F_DZ_INTERFACE, ICAR_F_QV};
    if (vars) {
        if (*n < 5) return fail(nullptr, ICAR_ADV_BAD_ARG, "vars needs room for 5 ids");
        memcpy(vars, set, sizeof(set));
    }
    *n = 5;
    return ICAR_ADV_OK;
}

int icar_adv_download(icar_adv_t *h, int32_t n, const int32_t *fields, float *const *host)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (n < 0 || (n > 0 && (!fields || !host))) return fail(h, ICAR_ADV_BAD_ARG, "bad field list");
    cudaSetDevice(h->desc.device);
    for (int f = 0; f < n; f++) {
        int e = copy_field(h, fields[f], host[f], nullptr, false, false);
        if (e) return e;
    }
    return icar_adv_sync(h);
}

int icar_adv_upload(icar_adv_t *h, int32_t n, const int32_t *fields, const float *const *host)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (n < 0 || (n > 0 && (!fields || !host))) return fail(h, ICAR_ADV_BAD_ARG, "bad field list");
    cudaSetDevice(h->desc.device);
    for (int f = 0; f < n; f++) {
        int e = copy_field(h, fields[f], const_cast<float *>(host[f]), nullptr, true);
        if (e) return e;
    }
    return icar_adv_sync(h);
}

static int device_copy(icar_adv_t *h, int32_t field, float *dev, bool to_handle)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (!dev) return fail(h, ICAR_ADV_BAD_ARG, "device pointer is NULL");
    cudaSetDevice(h->desc.device);
    FieldRef r;
    int e = resolve(h, field, r);
    if (e) return e;
    if (r.is_filter) return fail(h, ICAR_ADV_BAD_ARG, "the relaxation filter is set from host memory");
    const size_t P = (size_t)h->g.P;
    cudaError_t ce;
    if (to_handle)
        ce = cudaMemcpy2DAsync(r.buf->p, P * 4, dev, (size_t)r.ex * 4, (size_t)r.ex * 4, (size_t)r.ez * r.ey,
                               cudaMemcpyDeviceToDevice, h->stream);
    else
        ce = cudaMemcpy2DAsync(dev, (size_t)r.ex * 4, r.buf->p, P * 4, (size_t)r.ex * 4, (size_t)r.ez * r.ey,
                               cudaMemcpyDeviceToDevice, h->stream);
    if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaMemcpy2DAsync: %s", cudaGetErrorString(ce));
    if (to_handle) {
        if (r.flag) *r.flag = true;
        if (r.species >= 0 && !r.is_forcing && !r.is_dqdt) h->have_q[r.species] = true;
    }
    return ICAR_ADV_OK;
}

int icar_adv_set_field_device(icar_adv_t *h, int32_t field, const float *dev)
{
    return device_copy(h, field, const_cast<float *>(dev), true);
}

int icar_adv_get_field_device(icar_adv_t *h, int32_t field, float *dev) { return device_copy(h, field, dev, false); }

int icar_adv_advect(icar_adv_t *h, float dt)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (h->batch) return fail(h, ICAR_ADV_BAD_ARG, "domain is a batch member: step it with icar_adv_batch_step");
    cudaSetDevice(h->desc.device);
    return advect_impl(h, dt);
}

// apply_forcing for the species [s0, s1) that have forcing, in one launch.
static_assert(ICAR_ADV_MAX_SPECIES <= 32, "ForcingPtrs holds 32 species");
int forcing_range(icar_adv_t *h, double dt_seconds, int s0, int s1)
{
    if (h->nzone == 0) return ICAR_ADV_OK;
    icar::ForcingPtrs fp{};
    int ns = 0;
    for (int s = s0; s < s1; s++) {
        if (!h->forcing[s].p) continue;
        if (!h->dqdt[s].p) {
            int e = alloc(h, h->dqdt[s], h->n_cell);  // zero tendency: fixed inflow
            if (e) return e;
        }
        fp.q[ns] = h->q[s].p;
        fp.forcing[ns] = h->forcing[s].p;
        fp.dqdt[ns] = h->dqdt[s].p;
        ns++;
    }
    if (ns == 0) return ICAR_ADV_OK;
    const size_t n = (size_t)h->nzone * h->g.nz * ns;
    icar::k_apply_forcing<<<blocks_for(n, 256), 256, 0, h->stream>>>(h->g, h->nzone, h->zone_dev, h->filter_dev,
                                                                      dt_seconds, fp, ns);
    return check_launch(h, "apply_forcing");
}

int icar_adv_apply_forcing(icar_adv_t *h, double dt_seconds)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (h->batch) return fail(h, ICAR_ADV_BAD_ARG, "domain is a batch member: step it with icar_adv_batch_step");
    cudaSetDevice(h->desc.device);
    if (!std::isfinite(dt_seconds)) return fail(h, ICAR_ADV_BAD_ARG, "dt must be finite");
    return forcing_range(h, dt_seconds, 0, h->desc.n_species);
}

int icar_adv_enforce_limits(icar_adv_t *h)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    for (int s = 0; s < h->desc.n_species; s++)
        icar::k_enforce_limits<<<blocks_for(h->n_cell, 256), 256, 0, h->stream>>>(h->g, h->q[s].p);
    return check_launch(h, "enforce_limits", h->desc.n_species);
}

int icar_adv_balance_uvw(icar_adv_t *h)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (h->batch) return fail(h, ICAR_ADV_BAD_ARG, "domain is a batch member");
    cudaSetDevice(h->desc.device);
    const char *missing = nullptr;
    const int adv_den = h->opts.advect_density;
    if (!h->have_u) missing = "u";
    else if (!h->have_v) missing = "v";
    else if (!h->have_jac_u) missing = "jacobian_u";
    else if (!h->have_jac_v) missing = "jacobian_v";
    else if (!h->have_jac_w) missing = "jacobian_w";
    else if (!h->have_dz) missing = "advection_dz";
    else if (adv_den && !h->have_rho) missing = "density";
    if (missing) return fail(h, ICAR_ADV_NOT_READY, "field %s was never set", missing);
    const Geo &g = h->g;
    const float *rho = adv_den ? h->rho.p : h->jac.p;  // only read when advect_density
    const dim3 grid((unsigned)((g.nx + icar::balf::BX - 1) / icar::balf::BX),
                    (unsigned)((g.ny + icar::balf::BY - 1) / icar::balf::BY));
    icar::k_balance_uvw<<<grid, icar::balf::NT, icar::balf::SMEM, h->stream>>>(
        g, h->hs, h->desc.dx, adv_den, h->u.p, h->v.p, rho, h->dz.p, h->jac_u.p, h->jac_v.p, h->jac_w.p, h->w.p);
    h->have_w = true;
    return check_launch(h, "balance_uvw");
}

int icar_adv_compute_dt(icar_adv_t *h, const float *dz_levels, float cfl, int32_t cfl_strictness,
                        int32_t use_density, float *dt)
{
    if (!h || !dz_levels || !dt) return fail(h, ICAR_ADV_BAD_ARG, "NULL argument");
    if (cfl_strictness < 1 || cfl_strictness > 5) return fail(h, ICAR_ADV_BAD_ARG, "cfl_strictness must be 1..5");
    cudaSetDevice(h->desc.device);
    if (!h->have_u || !h->have_v || !h->have_w) return fail(h, ICAR_ADV_NOT_READY, "u, v and w must be set");
    const Geo &g = h->g;
    int e = alloc(h, h->dtbuf, 4 + (size_t)g.nz);
    if (e) return e;
    unsigned *d_out = reinterpret_cast<unsigned *>(h->dtbuf.p);
    float *d_dz = h->dtbuf.p + 4;
    CUDA_TRY(h, cudaMemcpyAsync(d_dz, dz_levels, sizeof(float) * g.nz, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemsetAsync(d_out, 0, 4 * sizeof(unsigned), h->stream));
    const size_t total = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
    const unsigned blocks = (unsigned)std::min<size_t>(blocks_for(total, 256), 148 * 8);
    icar::k_dt_maxima<<<blocks, 256, 0, h->stream>>>(g, h->hs, h->desc.dx, h->u.p, h->v.p, h->w.p, d_dz, d_out);
    e = check_launch(h, "compute_dt");
    if (e) return e;
    unsigned bits[4];
    CUDA_TRY(h, cudaMemcpyAsync(bits, d_out, sizeof(bits), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    float m[4];
    memcpy(m, bits, sizeof(m));
    *dt = icar::dt_from_maxima(m, cfl, cfl_strictness, use_density);
    if (*dt < 1e-1f)
        return fail(h, ICAR_ADV_CFL_VIOLATION, "time step too small: dt = %g s (max |u| %g, |v| %g, |w| %g)",
                    (double)*dt, (double)m[0], (double)m[1], (double)m[2]);
    return ICAR_ADV_OK;
}

int icar_adv_mp_simple(icar_adv_t *h, float dt)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (h->batch) return fail(h, ICAR_ADV_BAD_ARG, "domain is a batch member");
    if (!(dt >= 0.0f) || !std::isfinite(dt)) return fail(h, ICAR_ADV_BAD_ARG, "dt must be finite and >= 0");
    cudaSetDevice(h->desc.device);
    const int s_th = species_slot(h, ICAR_F_THETA), s_qv = species_slot(h, ICAR_F_QV),
              s_qc = species_slot(h, ICAR_F_QC), s_qr = species_slot(h, ICAR_F_QR), s_qs = species_slot(h, ICAR_F_QS);
    if (s_th < 0 || s_qv < 0 || s_qc < 0 || s_qr < 0 || s_qs < 0)
        return fail(h, ICAR_ADV_BAD_ARG, "mp_simple needs theta, qv, qc, qr and qs among the domain's fields");
    const char *missing = nullptr;
    if (!h->have_pressure) missing = "pressure";
    else if (!h->have_exner) missing = "exner";
    else if (!h->have_dz_mass) missing = "dz (dz_mass)";
    else if (!h->have_rho) missing = "density";
    else
        for (int s : {s_th, s_qv, s_qc, s_qr, s_qs})
            if (!h->have_q[s]) missing = "a microphysics species";
    if (missing) return fail(h, ICAR_ADV_NOT_READY, "field %s was never set", missing);
    const Geo &g = h->g;
    if (g.nz > 512) return fail(h, ICAR_ADV_BAD_ARG, "mp_simple supports at most 512 levels");
    const size_t n2 = (size_t)g.nx * g.ny;
    if (!h->acc_precip) {
        CUDA_TRY(h, dev_alloc(h, (void **)&h->acc_precip, 2 * n2 * sizeof(double)));
        CUDA_TRY(h, cudaMemsetAsync(h->acc_precip, 0, 2 * n2 * sizeof(double), h->stream));
    }
    if (!h->mp_stop) {
        CUDA_TRY(h, dev_alloc(h, (void **)&h->mp_stop, sizeof(int)));
        CUDA_TRY(h, cudaMemsetAsync(h->mp_stop, 0, sizeof(int), h->stream));
    }
    // the time constants of this dt, in the reference's FP32 (mp_simple.f90:618-622)
    const float cloud2snow = std::exp(-1.0f * (1.0f / 2000.0f) * dt);
    const float cloud2rain = std::exp(-1.0f * (1.0f / 500.0f) * dt);
    const int hs = h->hs;
    const int ti = std::max(g.nx - 2 * hs, 0), tj = std::max(g.ny - 2 * hs, 0);
    if (ti > 0 && tj > 0)
        icar::k_mp_simple<<<dim3((unsigned)((ti + icar::mpsf::BX - 1) / icar::mpsf::BX),
                                 (unsigned)((tj + icar::mpsf::BY - 1) / icar::mpsf::BY)),
                            icar::mpsf::NT, icar::mpsf::SMEM, h->stream>>>(
            g, hs, dt, cloud2rain, cloud2snow, h->pressure.p, h->q[s_th].p, h->exner.p, h->rho.p, h->q[s_qv].p,
            h->q[s_qc].p, h->q[s_qr].p, h->q[s_qs].p, h->dz_mass.p, h->acc_precip, h->acc_precip + n2, h->mp_stop);
    h->mp_ran = true;
    return check_launch(h, "mp_simple");
}

int icar_adv_get_precipitation(icar_adv_t *h, double *rain, double *snow)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    const size_t n2 = (size_t)h->g.nx * h->g.ny;
    if (!h->acc_precip) {
        if (rain) std::fill(rain, rain + n2, 0.0);
        if (snow) std::fill(snow, snow + n2, 0.0);
        return ICAR_ADV_OK;
    }
    if (rain) CUDA_TRY(h, cudaMemcpyAsync(rain, h->acc_precip, n2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (snow)
        CUDA_TRY(h, cudaMemcpyAsync(snow, h->acc_precip + n2, n2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    return icar_adv_sync(h);
}

int icar_adv_set_precipitation(icar_adv_t *h, const double *rain, const double *snow)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    const size_t n2 = (size_t)h->g.nx * h->g.ny;
    if (!h->acc_precip) CUDA_TRY(h, dev_alloc(h, (void **)&h->acc_precip, 2 * n2 * sizeof(double)));
    for (int part = 0; part < 2; part++) {
        const double *src = part == 0 ? rain : snow;
        double *dst = h->acc_precip + part * n2;
        if (src)
            CUDA_TRY(h, cudaMemcpyAsync(dst, src, n2 * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        else
            CUDA_TRY(h, cudaMemsetAsync(dst, 0, n2 * sizeof(double), h->stream));
    }
    return icar_adv_sync(h);
}

namespace {

// Species groups of icar_adv_step_host: one species per group up to 12 (on
// config 2 the step then runs within about 10 % of the page-locked copy
// time; 4 groups left 20 % more exposed).
constexpr int IO_GROUPS = 12;

int copy_species_async(icar_adv_t *h, float *dev, float *host, bool to_device, cudaStream_t st)
{
    const size_t P = (size_t)h->g.P, ex = (size_t)h->g.nx, rows = (size_t)h->g.nz * h->g.ny;
    cudaError_t ce = to_device ? cudaMemcpy2DAsync(dev, P * 4, host, ex * 4, ex * 4, rows, cudaMemcpyHostToDevice, st)
                               : cudaMemcpy2DAsync(host, ex * 4, dev, P * 4, ex * 4, rows, cudaMemcpyDeviceToHost, st);
    if (ce != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "cudaMemcpy2DAsync: %s", cudaGetErrorString(ce));
    return ICAR_ADV_OK;
}

}  // namespace

int icar_adv_step_host(icar_adv_t *h, double dt_seconds, int32_t enforce_limits, const float *const *q_in,
                       float *const *q_out)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (h->batch) return fail(h, ICAR_ADV_BAD_ARG, "domain is a batch member: step it with icar_adv_batch_step");
    const int S = h->desc.n_species;
    if (S > 0 && (!q_in || !q_out)) return fail(h, ICAR_ADV_BAD_ARG, "species pointer list is NULL");
    for (int s = 0; s < S; s++)
        if (!q_in[s] || !q_out[s]) return fail(h, ICAR_ADV_BAD_ARG, "species %d host pointer is NULL", s);
    if (!std::isfinite(dt_seconds)) return fail(h, ICAR_ADV_BAD_ARG, "dt must be finite");
    cudaSetDevice(h->desc.device);
    const bool mp = h->opts.advection == ICAR_ADV_MPDATA;
    const bool fused_mp = mp && !h->opts.rk3 && icar::fused_eligible(h->opts.mpdata_order, h->opts.mpdata_fct);
    int e;
    if (h->path == 1 || !(fused_mp || !mp) || h->opts.debug || S == 0) {
        // the unpipelined sequence (staged kernels, debug checks, RK3 MPDATA)
        for (int s = 0; s < S; s++)
            if ((e = copy_field(h, h->desc.species[s], const_cast<float *>(q_in[s]), nullptr, true))) return e;
        if ((e = icar_adv_step(h, dt_seconds, enforce_limits))) return e;
        for (int s = 0; s < S; s++)
            if ((e = copy_field(h, h->desc.species[s], q_out[s], nullptr, false, false))) return e;
        return icar_adv_sync(h);
    }
    const int ngroups = std::min(S, IO_GROUPS);
    if (!h->io_in) {
        CUDA_TRY(h, cudaStreamCreateWithFlags(&h->io_in, cudaStreamNonBlocking));
        CUDA_TRY(h, cudaStreamCreateWithFlags(&h->io_out, cudaStreamNonBlocking));
        h->io_events.assign(2 * IO_GROUPS + 1, nullptr);
        for (auto &ev : h->io_events) CUDA_TRY(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    // Every return after the first enqueue goes through `pipeline`, so that
    // on an error the copies already queued into or out of the caller's host
    // arrays are drained before the call returns.
    auto pipeline = [&]() -> int {
        cudaEvent_t ev_start = h->io_events[2 * IO_GROUPS];
        // uploads start once the work already queued on the handle's stream is done
        CUDA_TRY(h, cudaEventRecord(ev_start, h->stream));
        CUDA_TRY(h, cudaStreamWaitEvent(h->io_in, ev_start, 0));
        for (int s = 0; s < S; s++) h->have_q[s] = true;
        if ((e = ensure_ready(h))) return e;
        const float dt = (float)dt_seconds;
        if ((e = mp ? mpdata_prep(h, dt) : std_prep(h, dt))) return e;
        cudaEvent_t ev0 = nullptr, ev1 = nullptr;
        int64_t before = h->launches;
        if (h->profiling) {
            cudaEventCreate(&ev0);
            cudaEventCreate(&ev1);
            cudaEventRecord(ev0, h->stream);
        }
        auto result = [&](int s) -> DevBuf & { return mp ? h->qn[s] : (h->opts.rk3 ? h->q1s[s] : h->qn[s]); };
        for (int gi = 0; gi < ngroups; gi++) {
            const int s0 = S * gi / ngroups, s1 = S * (gi + 1) / ngroups;
            cudaEvent_t ev_in = h->io_events[gi], ev_done = h->io_events[IO_GROUPS + gi];
            for (int s = s0; s < s1; s++)
                if ((e = copy_species_async(h, h->q[s].p, const_cast<float *>(q_in[s]), true, h->io_in))) return e;
            CUDA_TRY(h, cudaEventRecord(ev_in, h->io_in));
            CUDA_TRY(h, cudaStreamWaitEvent(h->stream, ev_in, 0));
            if ((e = forcing_range(h, dt_seconds, s0, s1))) return e;
            if ((e = mp ? (h->path >= 2 ? mpdata_onepass_group(h, s0, s1) : mpdata_group(h, s0, s1))
                    : std_group(h, s0, s1)))
            return e;
            if (enforce_limits) {
                for (int s = s0; s < s1; s++)
                    icar::k_enforce_limits<<<blocks_for(h->n_cell, 256), 256, 0, h->stream>>>(h->g, result(s).p);
                if ((e = check_launch(h, "enforce_limits", s1 - s0))) return e;
            }
            CUDA_TRY(h, cudaEventRecord(ev_done, h->stream));
            CUDA_TRY(h, cudaStreamWaitEvent(h->io_out, ev_done, 0));
            for (int s = s0; s < s1; s++)
                if ((e = copy_species_async(h, result(s).p, q_out[s], false, h->io_out))) return e;
        }
        if (h->profiling) {
            cudaEventRecord(ev1, h->stream);
            h->events.emplace_back(ev0, ev1);
            h->timed_launches += h->launches - before;
        }
        CUDA_TRY(h, cudaStreamSynchronize(h->io_out));
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        for (int s = 0; s < S; s++) std::swap(h->q[s], result(s));
        return ICAR_ADV_OK;
    };
    if ((e = pipeline())) {
        cudaStreamSynchronize(h->io_in);
        cudaStreamSynchronize(h->io_out);
        cudaStreamSynchronize(h->stream);
        return e;
    }
    return icar_adv_sync(h);
}

int icar_adv_step(icar_adv_t *h, double dt_seconds, int32_t enforce_limits)
{
    int e = icar_adv_apply_forcing(h, dt_seconds);
    if (e) return e;
    e = icar_adv_advect(h, (float)dt_seconds);
    if (e) return e;
    if (enforce_limits) return icar_adv_enforce_limits(h);
    return ICAR_ADV_OK;
}

// After a sync: report (once) a tile whose TMA wait gave up in the
// single-pass kernel.
int check_op_err(icar_adv_t *h)
{
    if (!h->op_err) return ICAR_ADV_OK;
    int flag = 0;
    CUDA_TRY(h, cudaMemcpy(&flag, h->op_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!flag) return ICAR_ADV_OK;
    CUDA_TRY(h, cudaMemset(h->op_err, 0, sizeof(int)));
    if (flag == 2)
        return fail(h, ICAR_ADV_CUDA_ERROR, "single-pass MPDATA kernel: a TMA operand was misaligned (loads skipped)");
    return fail(h, ICAR_ADV_TIMEOUT, "a tile of the single-pass MPDATA kernel gave up waiting for its TMA loads");
}

int icar_adv_sync(icar_adv_t *h)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "stream sync: %s", cudaGetErrorString(e));
    int r = check_op_err(h);
    if (r) return r;
    return check_mp_stop(h);
}

}  // extern "C"

namespace {
// Poll a stream until its work is done or `timeout_s` seconds have passed;
// returns cudaSuccess, cudaErrorNotReady on timeout, or the stream's error.
cudaError_t wait_stream(cudaStream_t st, double timeout_s)
{
    const auto t0 = std::chrono::steady_clock::now();
    for (unsigned n = 0;; n++) {
        cudaError_t e = cudaStreamQuery(st);
        if (e != cudaErrorNotReady) return e;
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (el >= timeout_s) return cudaErrorNotReady;
        if (n > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}
}  // namespace

extern "C" {

int icar_adv_sync_timeout(icar_adv_t *h, double timeout_s)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (!(timeout_s >= 0.0)) return fail(h, ICAR_ADV_BAD_ARG, "timeout must be >= 0 seconds");
    cudaSetDevice(h->desc.device);
    cudaError_t e = wait_stream(h->stream, timeout_s);
    if (e == cudaErrorNotReady)
        return fail(h, ICAR_ADV_TIMEOUT, "the handle's work did not finish within %.3f s (it is still queued)",
                    timeout_s);
    if (e != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "stream sync: %s", cudaGetErrorString(e));
    return check_mp_stop(h);
}

int icar_adv_set_stream(icar_adv_t *h, void *cuda_stream)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaStream_t next = cuda_stream ? (cudaStream_t)cuda_stream : h->own_stream;
    if (next != h->stream) {
        // the handle's work stays in order across the switch: the new stream
        // waits for what is queued on the old one (no host wait)
        cudaSetDevice(h->desc.device);
        cudaEvent_t ev = nullptr;
        CUDA_TRY(h, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        cudaError_t e = cudaEventRecord(ev, h->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(next, ev, 0);
        cudaEventDestroy(ev);
        if (e != cudaSuccess) return fail(h, ICAR_ADV_CUDA_ERROR, "stream switch: %s", cudaGetErrorString(e));
    }
    h->stream = next;
    return ICAR_ADV_OK;
}

int icar_adv_device_bytes(const icar_adv_t *h, int64_t *bytes)
{
    if (!h || !bytes) return fail(nullptr, ICAR_ADV_BAD_ARG, "NULL argument");
    *bytes = (int64_t)h->bytes;
    return ICAR_ADV_OK;
}

const char *icar_adv_last_error(const icar_adv_t *h)
{
    if (!h) return g_create_error.c_str();
    return h->err.c_str();
}

int icar_adv_profile(icar_adv_t *h, int32_t enable)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    cudaStreamSynchronize(h->stream);
    for (auto *v : {&h->events, &h->corr_events}) {
        for (auto &p : *v) {
            cudaEventDestroy(p.first);
            cudaEventDestroy(p.second);
        }
        v->clear();
    }
    h->profiling = enable != 0;
    h->launches = 0;
    h->timed_launches = 0;
    return ICAR_ADV_OK;
}

int icar_adv_profile_read(icar_adv_t *h, double *species_kernel_ms, int64_t *species_kernel_launches,
                          int64_t *all_launches, int64_t *species_passes)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    double ms = 0.0;
    for (auto &p : h->events) {
        float t = 0.0f;
        CUDA_TRY(h, cudaEventElapsedTime(&t, p.first, p.second));
        ms += t;
    }
    if (species_kernel_ms) *species_kernel_ms = ms;
    if (species_kernel_launches) *species_kernel_launches = h->timed_launches;
    if (all_launches) *all_launches = h->launches;
    if (species_passes) *species_passes = (int64_t)h->events.size();
    return ICAR_ADV_OK;
}

int icar_adv_profile_read_correction(icar_adv_t *h, double *ms, int64_t *launches)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    cudaSetDevice(h->desc.device);
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    double total = 0.0;
    for (auto &p : h->corr_events) {
        float t = 0.0f;
        CUDA_TRY(h, cudaEventElapsedTime(&t, p.first, p.second));
        total += t;
    }
    if (ms) *ms = total;
    if (launches) *launches = (int64_t)h->corr_events.size();
    return ICAR_ADV_OK;
}

int icar_adv_set_tile_shape(icar_adv_t *h, int32_t shape)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (shape < 0 || shape >= icar::MP_NSHAPES) return fail(h, ICAR_ADV_BAD_ARG, "tile shape %d out of range", shape);
    h->mp_shape = shape;
    return ICAR_ADV_OK;
}

int icar_adv_set_species_group(icar_adv_t *h, int32_t group)
{
    if (!h) return fail(nullptr, ICAR_ADV_BAD_ARG, "handle is NULL");
    if (group < 0 || group > ICAR_ADV_MAX_SPECIES) return fail(h, ICAR_ADV_BAD_ARG, "species group %d out of range", group);
    h->sp_group = group;
    return ICAR_ADV_OK;
}

int icar_adv_tile_shapes(int32_t *n_shapes, int32_t *rows)
{
    if (!n_shapes) return fail(nullptr, ICAR_ADV_BAD_ARG, "NULL argument");
    if (rows && *n_shapes >= icar::MP_NSHAPES)
        for (int i = 0; i < icar::MP_NSHAPES; i++) rows[i] = icar::mp_shape_ty(i);
    *n_shapes = icar::MP_NSHAPES;
    return ICAR_ADV_OK;
}

// Internal selector used by the tests and the benchmark to run the staged
// kernels instead of the fused one (0 = fused when eligible, 1 = staged).
int icar_adv_set_path(icar_adv_t *h, int32_t path)
{
    if (!h || path < 0 || path > 3) return fail(h, ICAR_ADV_BAD_ARG, "bad path");
    h->path = path;
    return ICAR_ADV_OK;
}

}  // extern "C"

// ===========================================================================
// Batched form
// ===========================================================================
struct icar_adv_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    int nsm = 0;
    std::vector<icar_adv_t *> members;
    std::vector<double> dts;
    int shape = 1;
    int sp_group = 0;  // species per thread of the upwind pass (0 = all)
    int fct = -1;
    bool tables_dirty = true, graph_dirty = true;
    int parity = 0;
    // device tables and work lists
    icar::BatchMember *d_mem[2] = {nullptr, nullptr};
    size_t mem_cap = 0;
    int *d_ints = nullptr;   // prep prefix | upwind prefix | forcing prefix | counter
    size_t ints_cap = 0;
    int2 *d_pairs = nullptr;
    size_t pairs_cap = 0;
    int4 *d_items = nullptr;
    size_t items_cap = 0;
    int n_prep = 0, n_up = 0, n_force = 0, n_pairs = 0, n_items = 0, ctas = 0;
    // single-pass kernel (path 2 exact, 3 fast; 0 = the two-pass kernels):
    // per-member kernel parameters for both buffer parities, their TMA
    // descriptor tables, and one timeout flag for the whole batch
    int path = 0;
    icar::OnePassParams *d_opp[2] = {nullptr, nullptr};
    size_t opp_cap = 0;
    CUtensorMap *d_bmaps = nullptr;
    size_t bmaps_cap = 0;
    int *d_operr = nullptr;
    size_t off_up = 0, off_f = 0, off_counter = 0;
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    int stable_steps = 0;  // steps since the last table rebuild; graphs are captured once it reaches 2
    // pinned staging for the table uploads, two sets used in turn; an event
    // marks when a set's last upload has been consumed by the stream
    char *stage[2] = {nullptr, nullptr};
    size_t stage_cap[2] = {0, 0};
    cudaEvent_t stage_done[2] = {nullptr, nullptr};
    int stage_turn = 0;
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    int64_t steps = 0;
    std::string err;
};

namespace {

void batch_fields_changed(icar_adv_batch *b) { b->tables_dirty = b->graph_dirty = true; }

int bfail(icar_adv_batch_t *b, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (b)
        b->err = buf;
    else
        g_create_error = buf;
    return code;
}

#define BCUDA(b, call)                                                                              \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? ICAR_ADV_OOM : ICAR_ADV_CUDA_ERROR, \
                         "%s failed: %s", #call, cudaGetErrorString(e_));                           \
    } while (0)

template <class T>
int grow(icar_adv_batch_t *b, T *&p, size_t &cap, size_t n)
{
    if (n <= cap && p) return ICAR_ADV_OK;
    if (p) cudaFree(p);  // synchronises the device: queued launches may still read it
    p = nullptr;
    size_t c = std::max<size_t>(n + n / 2, 16);
    BCUDA(b, cudaMalloc(&p, c * sizeof(T)));
    cap = c;
    return ICAR_ADV_OK;
}

void drop_graphs(icar_adv_batch_t *b)
{
    for (int p = 0; p < 2; p++) {
        if (b->exec[p]) cudaGraphExecDestroy(b->exec[p]);
        if (b->graph[p]) cudaGraphDestroy(b->graph[p]);
        b->exec[p] = nullptr;
        b->graph[p] = nullptr;
    }
}

void fill_member(icar::BatchMember &m, icar_adv_t *h, double dt, int parity)
{
    memset(&m, 0, sizeof(m));
    m.g = h->g;
    m.dx = h->desc.dx;
    m.dt = (float)dt;
    m.dtd = dt;
    m.S = h->desc.n_species;
    m.adv_den = h->opts.advect_density;
    m.nzone = h->nzone;
    m.u = h->u.p; m.v = h->v.p; m.w = h->w.p; m.rho = h->rho.p; m.jac = h->jac.p;
    m.ju = h->jac_u.p; m.jv = h->jac_v.p; m.jw = h->jac_w.p; m.dz = h->dz.p;
    m.Um = h->Um.p; m.Vm = h->Vm.p; m.Wm = h->Wm.p; m.Gc = h->Gc.p; m.DJR = h->DJR.p; m.Wp = h->Wp.p;
    m.filter = h->filter_dev;
    m.zone = h->zone_dev;
    for (int s = 0; s < m.S; s++) {
        // parity 0: current state in q, next in qn; parity 1 the other way round
        float *cur = parity == 0 ? h->q[s].p : h->qn[s].p;
        float *nxt = parity == 0 ? h->qn[s].p : h->q[s].p;
        m.q0[s] = cur;
        m.out[s] = nxt;
        m.q1[s] = s < (int)h->q1s.size() ? h->q1s[s].p : nullptr;
        m.forcing[s] = h->forcing[s].p;
        m.dqdt[s] = h->dqdt[s].p;
    }
}

// Rebuild the member tables (both buffer parities) and the work lists.
int build_tables(icar_adv_batch_t *b)
{
    const int M = (int)b->members.size();
    std::vector<icar::BatchMember> mem[2];
    mem[0].resize(std::max(M, 1));
    mem[1].resize(std::max(M, 1));
    std::vector<int> prep(M + 1, 0), up(M + 1, 0), fpre(1, 0);
    std::vector<int2> pairs;
    std::vector<int4> items;
    const int ty = icar::mp_shape_ty(b->shape);
    const bool onepass = b->path >= 2;
    std::vector<icar::OnePassParams> opp[2];
    std::vector<CUtensorMap> maps;
    std::vector<size_t> map_base[2];
    if (onepass) {
        opp[0].resize(std::max(M, 1));
        opp[1].resize(std::max(M, 1));
        map_base[0].resize(M);
        map_base[1].resize(M);
        if (!b->d_operr) {
            BCUDA(b, cudaMalloc(&b->d_operr, sizeof(int)));
            BCUDA(b, cudaMemsetAsync(b->d_operr, 0, sizeof(int), b->stream));
        }
    }
    for (int m = 0; m < M; m++) {
        icar_adv_t *h = b->members[m];
        if (onepass) {
            int r = ensure_onepass(h);
            if (r) return bfail(b, r, "member scratch: %s", h->err.c_str());
            // descriptors of both parities: species inputs, then U_m, V_m, W_m/dz, J*rho
            for (int pp = 0; pp < 2; pp++) {
                map_base[pp][m] = maps.size();
                const int S = h->desc.n_species;
                for (int f = 0; f < S + 4; f++) {
                    const float *base = f < S ? (pp == 0 ? h->q[f].p : h->qn[f].p)
                                              : (f == S ? h->Um.p : f == S + 1 ? h->Vm.p : f == S + 2 ? h->Wp.p : h->Gc.p);
                    const CUtensorMap *mp;
                    if ((r = plane_map(h, base, f == S + 1 ? h->g.ny + 1 : h->g.ny, &mp)))
                        return bfail(b, r, "%s", h->err.c_str());
                    maps.push_back(*mp);
                }
            }
        } else {
            int r = ensure_fused(h);
            if (r) return bfail(b, r, "member scratch: %s", h->err.c_str());
        }
        // members' buffers hold "current" in q at the batch's parity 0
        fill_member(mem[0][m], h, b->dts[m], b->parity == 0 ? 0 : 1);
        fill_member(mem[1][m], h, b->dts[m], b->parity == 0 ? 1 : 0);
        const Geo &g = h->g;
        const size_t nf = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
        prep[m + 1] = prep[m] + (int)((nf + 255) / 256);
        up[m + 1] = up[m] + icar::upwind_cols_blocks(h->g, h->desc.n_species, b->sp_group);
        for (int s = 0; s < h->desc.n_species; s++) {
            if (h->forcing[s].p && h->nzone > 0) {
                pairs.push_back(make_int2(m, s));
                fpre.push_back(fpre.back() + (int)(((size_t)h->nzone * g.nz + 255) / 256));
            }
        }
        if (onepass) {
            const int tx = onepass_tiles_x(g), tyn = onepass_tiles_y(g);
            for (int s = 0; s < h->desc.n_species; s++)
                for (int a = 0; a < tyn; a++)
                    for (int c = 0; c < tx; c++)
                        items.push_back(make_int4(m, s, c, a * icar::op::TY));
        } else {
            const int tx = icar::mp_tiles_x(g), tyn = icar::mp_tiles_y(g, ty);
            for (int s = 0; s < h->desc.n_species; s++)
                for (int a = 0; a < tyn; a++)
                    for (int c = 0; c < tx; c++)
                        items.push_back(make_int4(m, s, c * icar::mpf::TX - 2, 1 + a * ty));
        }
    }
    if (onepass && !maps.empty() && (maps.size() > b->bmaps_cap || !b->d_bmaps)) {
        if (b->d_bmaps) cudaFree(b->d_bmaps);  // synchronises: queued launches may read it
        b->d_bmaps = nullptr;
        b->bmaps_cap = 0;
        const size_t cap = maps.size() * 3 / 2 + 16;
        BCUDA(b, cudaMalloc(&b->d_bmaps, cap * sizeof(CUtensorMap)));
        b->bmaps_cap = cap;
    }
    if (onepass) {
        for (int pp = 0; pp < 2; pp++)
            for (int m = 0; m < M; m++) {
                icar_adv_t *h = b->members[m];
                icar::OnePassParams &q = opp[pp][m];
                memset(&q, 0, sizeof(q));
                const int S = h->desc.n_species;
                q.q0maps = b->d_bmaps + map_base[pp][m];
                q.fmaps = q.q0maps + S;
                for (int s2 = 0; s2 < S; s2++) q.out[s2] = pp == 0 ? h->qn[s2].p : h->q[s2].p;
                q.Wm = h->Wm.p;
                q.DJR = h->DJR.p;
                q.dz = h->dz.p;
                q.err = b->d_operr;
                q.g = h->g;
                q.nspecies = S;
                q.tiles_x = onepass_tiles_x(h->g);
            }
        if ((size_t)std::max(M, 1) > b->opp_cap || !b->d_opp[0]) {
            for (int pp = 0; pp < 2; pp++) {
                if (b->d_opp[pp]) cudaFree(b->d_opp[pp]);
                b->d_opp[pp] = nullptr;
            }
            b->opp_cap = 0;
            const size_t cap = std::max<size_t>(M, 16);
            for (int pp = 0; pp < 2; pp++) BCUDA(b, cudaMalloc(&b->d_opp[pp], cap * sizeof(icar::OnePassParams)));
            b->opp_cap = cap;
        }
    }
    // longest columns first (cost ~ nz per tile), so the tail of the
    // launch is made of short items
    std::stable_sort(items.begin(), items.end(), [&](const int4 &x, const int4 &y) {
        return b->members[x.x]->g.nz > b->members[y.x]->g.nz;
    });
    b->n_prep = prep[M];
    b->n_up = up[M];
    b->n_pairs = (int)pairs.size();
    b->n_force = fpre.back();
    b->n_items = (int)items.size();
    int e;
    if ((size_t)std::max(M, 1) > b->mem_cap || !b->d_mem[0]) {
        for (int p = 0; p < 2; p++) {
            if (b->d_mem[p]) cudaFree(b->d_mem[p]);
            b->d_mem[p] = nullptr;
        }
        b->mem_cap = 0;
        const size_t cap = std::max<size_t>(M, 16);
        for (int p = 0; p < 2; p++) BCUDA(b, cudaMalloc(&b->d_mem[p], cap * sizeof(icar::BatchMember)));
        b->mem_cap = cap;
    }
    b->off_up = M + 1;
    b->off_f = b->off_up + M + 1;
    b->off_counter = b->off_f + fpre.size();
    std::vector<int> ints(b->off_counter + 1, 0);
    std::copy(prep.begin(), prep.end(), ints.begin());
    std::copy(up.begin(), up.end(), ints.begin() + b->off_up);
    std::copy(fpre.begin(), fpre.end(), ints.begin() + b->off_f);
    if ((e = grow(b, b->d_ints, b->ints_cap, ints.size()))) return e;
    if ((e = grow(b, b->d_pairs, b->pairs_cap, std::max<size_t>(pairs.size(), 1)))) return e;
    if ((e = grow(b, b->d_items, b->items_cap, std::max<size_t>(items.size(), 1)))) return e;
    // Upload through pinned staging, stream-ordered after every launch already
    // queued (those still read the old tables), without a host sync.  Two
    // staging sets alternate; a set is reused only after its previous upload
    // has been consumed.
    const size_t bm = sizeof(icar::BatchMember) * std::max(M, 1);
    const size_t po = onepass ? sizeof(icar::OnePassParams) * std::max(M, 1) : 0;
    const size_t seg[8] = {bm, bm, sizeof(int) * ints.size(), sizeof(int2) * pairs.size(),
                           sizeof(int4) * items.size(), po, po, sizeof(CUtensorMap) * maps.size()};
    size_t off[8], total = 0;
    for (int i = 0; i < 8; i++) {
        off[i] = total;
        total += (seg[i] + 255) / 256 * 256;
    }
    const int t = b->stage_turn;
    if (b->stage_done[t]) BCUDA(b, cudaEventSynchronize(b->stage_done[t]));
    else BCUDA(b, cudaEventCreateWithFlags(&b->stage_done[t], cudaEventDisableTiming));
    if (total > b->stage_cap[t]) {
        if (b->stage[t]) cudaFreeHost(b->stage[t]);
        b->stage[t] = nullptr;
        b->stage_cap[t] = 0;
        BCUDA(b, cudaHostAlloc((void **)&b->stage[t], total * 3 / 2, cudaHostAllocDefault));
        b->stage_cap[t] = total * 3 / 2;
    }
    char *st = b->stage[t];
    memcpy(st + off[0], mem[0].data(), seg[0]);
    memcpy(st + off[1], mem[1].data(), seg[1]);
    memcpy(st + off[2], ints.data(), seg[2]);
    if (seg[3]) memcpy(st + off[3], pairs.data(), seg[3]);
    if (seg[4]) memcpy(st + off[4], items.data(), seg[4]);
    if (seg[5]) memcpy(st + off[5], opp[0].data(), seg[5]);
    if (seg[6]) memcpy(st + off[6], opp[1].data(), seg[6]);
    if (seg[7]) memcpy(st + off[7], maps.data(), seg[7]);
    BCUDA(b, cudaMemcpyAsync(b->d_mem[0], st + off[0], seg[0], cudaMemcpyHostToDevice, b->stream));
    BCUDA(b, cudaMemcpyAsync(b->d_mem[1], st + off[1], seg[1], cudaMemcpyHostToDevice, b->stream));
    BCUDA(b, cudaMemcpyAsync(b->d_ints, st + off[2], seg[2], cudaMemcpyHostToDevice, b->stream));
    if (seg[3]) BCUDA(b, cudaMemcpyAsync(b->d_pairs, st + off[3], seg[3], cudaMemcpyHostToDevice, b->stream));
    if (seg[4]) BCUDA(b, cudaMemcpyAsync(b->d_items, st + off[4], seg[4], cudaMemcpyHostToDevice, b->stream));
    if (seg[5]) BCUDA(b, cudaMemcpyAsync(b->d_opp[0], st + off[5], seg[5], cudaMemcpyHostToDevice, b->stream));
    if (seg[6]) BCUDA(b, cudaMemcpyAsync(b->d_opp[1], st + off[6], seg[6], cudaMemcpyHostToDevice, b->stream));
    if (seg[7]) BCUDA(b, cudaMemcpyAsync(b->d_bmaps, st + off[7], seg[7], cudaMemcpyHostToDevice, b->stream));
    BCUDA(b, cudaEventRecord(b->stage_done[t], b->stream));
    b->stage_turn ^= 1;
    // the single-pass launch has one CTA per item; the two-pass correction
    // kernel is persistent
    b->ctas = onepass ? b->n_items
                      : std::min(std::max(b->n_items, 1), icar::batch_corr_max_ctas(b->shape, b->fct, b->nsm));
    b->tables_dirty = false;
    return ICAR_ADV_OK;
}

// Enqueue one batched step using the member table of the given parity.
void enqueue_step(icar_adv_batch_t *b, int p, cudaStream_t st)
{
    const icar::BatchMember *mem = b->d_mem[p];
    const int M = (int)b->members.size();
    if (b->n_force > 0)
        icar::k_batch_forcing<<<b->n_force, 256, 0, st>>>(mem, b->d_ints + b->off_f, b->d_pairs, b->n_pairs);
    if (b->n_prep > 0) icar::k_batch_prep<<<b->n_prep, 256, 0, st>>>(mem, b->d_ints, M);
    if (b->path >= 2) {
        if (b->n_items > 0) {
            const icar::OnePassParams *opp = b->d_opp[p];
            const int n = b->n_items;
            const size_t sm = icar::op::SMEM;
            const int4 *it = b->d_items;
            if (b->path == 2 && b->fct) icar::k_batch_onepass_items<true, true><<<n, icar::op::NT, sm, st>>>(opp, it);
            else if (b->path == 2) icar::k_batch_onepass_items<true, false><<<n, icar::op::NT, sm, st>>>(opp, it);
            else if (b->fct) icar::k_batch_onepass_items<false, true><<<n, icar::op::NT, sm, st>>>(opp, it);
            else icar::k_batch_onepass_items<false, false><<<n, icar::op::NT, sm, st>>>(opp, it);
        }
        return;
    }
    if (b->n_up > 0)
        icar::k_batch_upwind<<<b->n_up, icar::upf::NT, icar::upf::SMEM, st>>>(mem, b->d_ints + b->off_up, M,
                                                                           b->sp_group);
    cudaMemsetAsync(b->d_ints + b->off_counter, 0, sizeof(int), st);
    if (b->n_items > 0)
        icar::batch_corr_launch(st, b->shape, b->ctas, b->fct, mem, b->d_items, b->n_items,
                                b->d_ints + b->off_counter);
}

cudaError_t batch_onepass_setup()
{
    const int sm = (int)icar::op::SMEM;
    cudaError_t e =
        cudaFuncSetAttribute(icar::k_batch_onepass_items<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(icar::k_batch_onepass_items<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(icar::k_batch_onepass_items<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(icar::k_batch_onepass_items<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
    return e;
}

int build_graphs(icar_adv_batch_t *b)
{
    drop_graphs(b);
    for (int p = 0; p < 2; p++) {
        BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(b, p, b->stream);
        cudaError_t e = cudaStreamEndCapture(b->stream, &b->graph[p]);
        if (e != cudaSuccess) return bfail(b, ICAR_ADV_CUDA_ERROR, "graph capture failed: %s", cudaGetErrorString(e));
        BCUDA(b, cudaGraphInstantiate(&b->exec[p], b->graph[p], 0));
    }
    b->graph_dirty = false;
    return ICAR_ADV_OK;
}

}  // namespace

extern "C" {

int icar_adv_batch_create(int32_t device, icar_adv_batch_t **out)
{
    if (!out) return bfail(nullptr, ICAR_ADV_BAD_ARG, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return bfail(nullptr, ICAR_ADV_CUDA_ERROR, "device %d not available", device);
    cudaSetDevice(device);
    icar_adv_batch_t *b = new icar_adv_batch();
    b->device = device;
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = icar::mp_corr_setup();
    if (e == cudaSuccess) e = icar::batch_setup();
    if (e == cudaSuccess) e = batch_onepass_setup();
    if (e != cudaSuccess) {
        int code = bfail(nullptr, ICAR_ADV_CUDA_ERROR, "batch setup failed: %s", cudaGetErrorString(e));
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return code;
    }
    *out = b;
    return ICAR_ADV_OK;
}

int icar_adv_batch_add(icar_adv_batch_t *b, icar_adv_t *h, double dt_seconds)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    if (!h) return bfail(b, ICAR_ADV_BAD_ARG, "member is NULL");
    if (h->batch) return bfail(b, ICAR_ADV_BAD_ARG, "domain already belongs to a batch");
    if (h->desc.device != b->device) return bfail(b, ICAR_ADV_BAD_ARG, "member lives on another device");
    if (h->opts.advection != ICAR_ADV_MPDATA || h->opts.rk3 || !icar::fused_eligible(h->opts.mpdata_order, h->opts.mpdata_fct))
        return bfail(b, ICAR_ADV_BAD_ARG, "batched members must use MPDATA order 2 (with or without FCT), no RK3");
    if (b->fct >= 0 && b->fct != h->opts.mpdata_fct)
        return bfail(b, ICAR_ADV_BAD_ARG, "all members of a batch share the MPDATA_FCT switch");
    if (!(dt_seconds >= 0.0) || !std::isfinite(dt_seconds)) return bfail(b, ICAR_ADV_BAD_ARG, "dt must be finite, >= 0");
    cudaSetDevice(b->device);
    int e = ensure_ready(h);
    if (e) return bfail(b, e, "member not ready: %s", h->err.c_str());
    e = b->path >= 2 ? ensure_onepass(h) : ensure_fused(h);
    if (e) return bfail(b, e, "member scratch: %s", h->err.c_str());
    // order the member's pending work before the batch's, then share the stream
    cudaStreamSynchronize(h->stream);
    for (int s = 0; s < h->desc.n_species; s++)
        if (h->forcing[s].p && !h->dqdt[s].p) {
            e = alloc(h, h->dqdt[s], h->n_cell);
            if (e) return bfail(b, e, "%s", h->err.c_str());
        }
    cudaStreamSynchronize(h->stream);
    h->stream = b->stream;
    h->batch = b;
    b->fct = h->opts.mpdata_fct;
    b->members.push_back(h);
    b->dts.push_back(dt_seconds);
    b->tables_dirty = b->graph_dirty = true;
    return ICAR_ADV_OK;
}

int icar_adv_batch_remove(icar_adv_batch_t *b, icar_adv_t *h)
{
    if (!b || !h) return bfail(b, ICAR_ADV_BAD_ARG, "NULL argument");
    auto it = std::find(b->members.begin(), b->members.end(), h);
    if (it == b->members.end()) return bfail(b, ICAR_ADV_BAD_ARG, "domain is not a member of this batch");
    cudaSetDevice(b->device);
    // the member's own stream waits for every batch launch already queued
    // (they may still read its buffers); no host synchronisation
    cudaEvent_t ev = nullptr;
    BCUDA(b, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    BCUDA(b, cudaEventRecord(ev, b->stream));
    BCUDA(b, cudaStreamWaitEvent(h->own_stream, ev, 0));
    cudaEventDestroy(ev);
    b->dts.erase(b->dts.begin() + (it - b->members.begin()));
    b->members.erase(it);
    h->batch = nullptr;
    h->stream = h->own_stream;
    if (b->members.empty()) b->fct = -1;
    b->tables_dirty = b->graph_dirty = true;
    return ICAR_ADV_OK;
}

int icar_adv_batch_set_dt(icar_adv_batch_t *b, icar_adv_t *h, double dt_seconds)
{
    if (!b || !h) return bfail(b, ICAR_ADV_BAD_ARG, "NULL argument");
    auto it = std::find(b->members.begin(), b->members.end(), h);
    if (it == b->members.end()) return bfail(b, ICAR_ADV_BAD_ARG, "domain is not a member of this batch");
    if (!(dt_seconds >= 0.0) || !std::isfinite(dt_seconds)) return bfail(b, ICAR_ADV_BAD_ARG, "dt must be finite, >= 0");
    b->dts[it - b->members.begin()] = dt_seconds;
    b->tables_dirty = true;
    return ICAR_ADV_OK;
}

int icar_adv_batch_set_tile_shape(icar_adv_batch_t *b, int32_t shape)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    if (shape < 0 || shape >= icar::MP_NSHAPES) return bfail(b, ICAR_ADV_BAD_ARG, "tile shape out of range");
    if (shape != b->shape) {
        b->shape = shape;
        b->tables_dirty = b->graph_dirty = true;
    }
    return ICAR_ADV_OK;
}

int icar_adv_batch_set_species_group(icar_adv_batch_t *b, int32_t group)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    if (group < 0 || group > ICAR_ADV_MAX_SPECIES) return bfail(b, ICAR_ADV_BAD_ARG, "species group out of range");
    if (group != b->sp_group) {
        b->sp_group = group;
        b->tables_dirty = b->graph_dirty = true;
    }
    return ICAR_ADV_OK;
}

int icar_adv_batch_step(icar_adv_batch_t *b)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    cudaSetDevice(b->device);
    if (b->members.empty()) return ICAR_ADV_OK;
    int e;
    if (b->tables_dirty) {
        // tables are written relative to the current parity, so rebuild from parity 0
        b->parity = 0;
        if ((e = build_tables(b))) return e;
        b->graph_dirty = true;
        b->stable_steps = 0;
    }
    // while membership keeps changing (serving), launch directly; capture the
    // step in graphs once the same tables have served two steps
    if (b->graph_dirty && b->stable_steps >= 2 && (e = build_graphs(b))) return e;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    if (b->profiling) {
        cudaEventCreate(&ev0);
        cudaEventCreate(&ev1);
        cudaEventRecord(ev0, b->stream);
    }
    if (!b->graph_dirty) {
        BCUDA(b, cudaGraphLaunch(b->exec[b->parity], b->stream));
    } else {
        enqueue_step(b, b->parity, b->stream);
        BCUDA(b, cudaGetLastError());
    }
    b->stable_steps++;
    if (b->profiling) {
        cudaEventRecord(ev1, b->stream);
        b->events.emplace_back(ev0, ev1);
    }
    b->steps++;
    b->parity ^= 1;
    // the members' "current" buffers are now the ones just written
    for (icar_adv_t *h : b->members)
        for (int s = 0; s < h->desc.n_species; s++) std::swap(h->q[s], h->qn[s]);
    // keep the tables consistent with the swapped member buffers: parity p's
    // table reads q (current) when p == parity, which holds by construction
    // of build_tables (table[0] read q at parity 0, table[1] read qn) as the
    // buffers and the parity flip together.
    return ICAR_ADV_OK;
}

int icar_adv_batch_sync(icar_adv_batch_t *b)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    cudaSetDevice(b->device);
    BCUDA(b, cudaStreamSynchronize(b->stream));
    if (b->d_operr) {
        int flag = 0;
        BCUDA(b, cudaMemcpy(&flag, b->d_operr, sizeof(int), cudaMemcpyDeviceToHost));
        if (flag) {
            BCUDA(b, cudaMemset(b->d_operr, 0, sizeof(int)));
            return bfail(b, flag == 2 ? ICAR_ADV_CUDA_ERROR : ICAR_ADV_TIMEOUT,
                         flag == 2 ? "single-pass MPDATA kernel: a TMA operand was misaligned (loads skipped)"
                                   : "a tile of the single-pass MPDATA kernel gave up waiting for its TMA loads");
        }
    }
    return ICAR_ADV_OK;
}

int icar_adv_batch_set_path(icar_adv_batch_t *b, int32_t path)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    if (path != 0 && path != 2 && path != 3) return bfail(b, ICAR_ADV_BAD_ARG, "batch path must be 0, 2 or 3");
    if (path != b->path) {
        b->path = path;
        b->tables_dirty = b->graph_dirty = true;
    }
    return ICAR_ADV_OK;
}

int icar_adv_batch_sync_timeout(icar_adv_batch_t *b, double timeout_s)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    if (!(timeout_s >= 0.0)) return bfail(b, ICAR_ADV_BAD_ARG, "timeout must be >= 0 seconds");
    cudaSetDevice(b->device);
    cudaError_t e = wait_stream(b->stream, timeout_s);
    if (e == cudaErrorNotReady)
        return bfail(b, ICAR_ADV_TIMEOUT, "the batch's steps did not finish within %.3f s (still queued)", timeout_s);
    if (e != cudaSuccess) return bfail(b, ICAR_ADV_CUDA_ERROR, "stream sync: %s", cudaGetErrorString(e));
    return ICAR_ADV_OK;
}

int icar_adv_batch_set_stream(icar_adv_batch_t *b, void *cuda_stream)
{
    if (!b || !cuda_stream) return bfail(b, ICAR_ADV_BAD_ARG, "batch or stream is NULL");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    b->stream = (cudaStream_t)cuda_stream;
    for (icar_adv_t *h : b->members) h->stream = b->stream;
    b->graph_dirty = true;
    return ICAR_ADV_OK;
}

int icar_adv_batch_profile(icar_adv_batch_t *b, int32_t enable)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (auto &p : b->events) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    b->events.clear();
    b->profiling = enable != 0;
    return ICAR_ADV_OK;
}

int icar_adv_batch_profile_read(icar_adv_batch_t *b, double *step_ms, int64_t *steps, int64_t *kernels_per_step,
                                int64_t *cell_species_per_step)
{
    if (!b) return bfail(nullptr, ICAR_ADV_BAD_ARG, "batch is NULL");
    cudaSetDevice(b->device);
    BCUDA(b, cudaStreamSynchronize(b->stream));
    double ms = 0.0;
    for (auto &p : b->events) {
        float t = 0.0f;
        BCUDA(b, cudaEventElapsedTime(&t, p.first, p.second));
        ms += t;
    }
    if (step_ms) *step_ms = ms;
    if (steps) *steps = (int64_t)b->events.size();
    if (kernels_per_step)
        *kernels_per_step = (b->n_force > 0) + (b->n_prep > 0) + (b->n_up > 0) + (b->n_items > 0);
    if (cell_species_per_step) {
        int64_t cs = 0;
        for (icar_adv_t *h : b->members) cs += (int64_t)h->g.nx * h->g.ny * h->g.nz * h->desc.n_species;
        *cell_species_per_step = cs;
    }
    return ICAR_ADV_OK;
}

int icar_adv_batch_destroy(icar_adv_batch_t *b)
{
    if (!b) return ICAR_ADV_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    for (icar_adv_t *h : b->members) {
        h->batch = nullptr;
        h->stream = h->own_stream;
    }
    drop_graphs(b);
    for (auto &p : b->events) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    if (b->d_mem[0]) cudaFree(b->d_mem[0]);
    if (b->d_mem[1]) cudaFree(b->d_mem[1]);
    if (b->d_ints) cudaFree(b->d_ints);
    if (b->d_pairs) cudaFree(b->d_pairs);
    if (b->d_items) cudaFree(b->d_items);
    for (auto *q : b->d_opp)
        if (q) cudaFree(q);
    if (b->d_bmaps) cudaFree(b->d_bmaps);
    if (b->d_operr) cudaFree(b->d_operr);
    for (int t = 0; t < 2; t++) {
        if (b->stage[t]) cudaFreeHost(b->stage[t]);
        if (b->stage_done[t]) cudaEventDestroy(b->stage_done[t]);
    }
    cudaStreamDestroy(b->stream);
    delete b;
    return ICAR_ADV_OK;
}

const char *icar_adv_batch_last_error(const icar_adv_batch_t *b) { return b ? b->err.c_str() : g_create_error.c_str(); }

}  // extern "C"

// ===========================================================================
// MPDATA step into caller-owned device memory, allocating nothing
// ===========================================================================
// For callers that cannot allocate device memory themselves (see
// icar_adv_advect_noalloc in include/icar_adv.h).  The per-step scratch of
// the fused path (U_m, V_m, W_m, J*rho, dz*J*rho, W_m/dz and one pass-1
// field) lives in this file-scope array instead of cudaMalloc'ed buffers.
// Every GPU that loads the library holds it until the process exits, and
// every call on a device shares it.
namespace {

constexpr size_t NOALLOC_SCRATCH_FLOATS = (size_t)4 << 20;  // 4 Mi floats = 16 MiB per device
__device__ __align__(256) float g_noalloc_scratch[NOALLOC_SCRATCH_FLOATS];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mutex;
float *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};  // device address of g_noalloc_scratch, per device

// Once per device, with that device current: the array's device address (a
// host-side `g_noalloc_scratch` is only a stand-in symbol, not a pointer the
// kernels may use) and the fused kernel's shared-memory opt-in.
int noalloc_setup(int dev, float **out)
{
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        float *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(nullptr, ICAR_ADV_CUDA_ERROR, "cudaGetSymbolAddress of the static scratch failed: %s",
                        cudaGetErrorString(e));
        e = icar::mp_corr_setup();
        if (e != cudaSuccess)
            return fail(nullptr, ICAR_ADV_CUDA_ERROR, "kernel setup failed: %s", cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return ICAR_ADV_OK;
}

inline size_t round64(size_t n) { return (n + 63) / 64 * 64; }

}  // namespace

extern "C" int icar_adv_advect_noalloc(const icar_adv_noalloc_args *a)
{
    if (!a) return fail(nullptr, ICAR_ADV_BAD_ARG, "args is NULL");
    if (a->nx < 3 || a->ny < 3 || a->nz < 3)
        return fail(nullptr, ICAR_ADV_BAD_ARG, "domain %dx%dx%d too small (each extent must be >= 3)", a->nx, a->ny,
                    a->nz);
    if (a->n_species < 0 || a->n_species > ICAR_ADV_MAX_SPECIES)
        return fail(nullptr, ICAR_ADV_BAD_ARG, "n_species %d out of range", a->n_species);
    if (!(a->dx > 0.0f) || !std::isfinite(a->dx) || !(a->dt >= 0.0f) || !std::isfinite(a->dt))
        return fail(nullptr, ICAR_ADV_BAD_ARG, "dx must be positive and dt finite and >= 0");
    if (!a->u || !a->v || !a->w || !a->density || !a->jacobian || !a->jacobian_u || !a->jacobian_v ||
        !a->jacobian_w || !a->advection_dz)
        return fail(nullptr, ICAR_ADV_BAD_ARG, "a wind or metric field pointer is NULL");
    for (int s = 0; s < a->n_species; s++)
        if (!a->q_in[s] || !a->q_out[s]) return fail(nullptr, ICAR_ADV_BAD_ARG, "species %d pointer is NULL", s);
    Geo g;
    g.nx = a->nx;
    g.ny = a->ny;
    g.nz = a->nz;
    g.P = ((a->nx + 1) + 3) / 4 * 4;
    const size_t nc = (size_t)g.P * g.nz * g.ny, nv = (size_t)g.P * g.nz * (g.ny + 1);
    // U_m (nc), V_m (nv), then W_m, G, DJR, W', q1 (nc each), each 256-byte aligned
    const size_t need = round64(nc) * 6 + round64(nv);
    if (need > NOALLOC_SCRATCH_FLOATS)
        return fail(nullptr, ICAR_ADV_BAD_ARG,
                    "domain %dx%dx%d needs %zu floats of scratch; the static scratch holds %zu "
                    "(use the handle API, which allocates, for larger domains)",
                    a->nx, a->ny, a->nz, need, NOALLOC_SCRATCH_FLOATS);
    // The kernels stage whole rows with 16-byte asynchronous copies, so every
    // array must start on a 16-byte boundary (the pitched rows then do too).
    const void *inputs[9] = {a->u, a->v, a->w, a->density, a->jacobian, a->jacobian_u, a->jacobian_v,
                             a->jacobian_w, a->advection_dz};
    const char *input_names[9] = {"u", "v", "w", "density", "jacobian", "jacobian_u", "jacobian_v", "jacobian_w",
                                  "advection_dz"};
    for (int f = 0; f < 9; f++)
        if ((uintptr_t)inputs[f] & 15u)
            return fail(nullptr, ICAR_ADV_BAD_ARG, "%s is not 16-byte aligned", input_names[f]);
    for (int s = 0; s < a->n_species; s++)
        if (((uintptr_t)a->q_in[s] | (uintptr_t)a->q_out[s]) & 15u)
            return fail(nullptr, ICAR_ADV_BAD_ARG, "species %d: q_in and q_out must be 16-byte aligned", s);
    // Species run one after another on one stream, so an output that
    // overlaps any input (or another output) would silently feed updated
    // values into a later species: refuse every overlap.
    auto overlaps = [](const void *p, size_t np, const void *q, size_t nq) {
        const uintptr_t a0 = (uintptr_t)p, b0 = (uintptr_t)q;
        return a0 < b0 + nq * sizeof(float) && b0 < a0 + np * sizeof(float);
    };
    const size_t n_in[9] = {nc, nv, nc, nc, nc, nc, nv, nc, nc};
    for (int s = 0; s < a->n_species; s++) {
        for (int t = 0; t < a->n_species; t++) {
            if (overlaps(a->q_out[s], nc, a->q_in[t], nc))
                return fail(nullptr, ICAR_ADV_BAD_ARG, "q_out[%d] overlaps q_in[%d] (no aliasing)", s, t);
            if (t != s && overlaps(a->q_out[s], nc, a->q_out[t], nc))
                return fail(nullptr, ICAR_ADV_BAD_ARG, "q_out[%d] overlaps q_out[%d] (no aliasing)", s, t);
        }
        for (int f = 0; f < 9; f++)
            if (overlaps(a->q_out[s], nc, inputs[f], n_in[f]))
                return fail(nullptr, ICAR_ADV_BAD_ARG, "q_out[%d] overlaps %s (no aliasing)", s, input_names[f]);
    }
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
        return fail(nullptr, ICAR_ADV_CUDA_ERROR, "no usable current device: %s", cudaGetErrorString(ce));
    float *base = nullptr;
    int e = noalloc_setup(dev, &base);
    if (e) return e;
    cudaStream_t st = (cudaStream_t)a->stream;
    float *Um = base, *Vm = Um + round64(nc), *Wm = Vm + round64(nv), *Gc = Wm + round64(nc),
          *DJR = Gc + round64(nc), *Wp = DJR + round64(nc), *q1 = Wp + round64(nc);
    // the array keeps the previous call's contents; the padding columns the
    // tile loads read must start at zero, so clear the part this call uses
    ce = cudaMemsetAsync(base, 0, need * sizeof(float), st);
    if (ce != cudaSuccess) return fail(nullptr, ICAR_ADV_CUDA_ERROR, "cudaMemsetAsync: %s", cudaGetErrorString(ce));
    const size_t nf = (size_t)(g.nx + 1) * g.nz * (g.ny + 1);
    icar::k_mp_prep<<<blocks_for(nf, 256), 256, 0, st>>>(g, a->dx, a->dt, a->advect_density, a->u, a->v, a->w,
                                                       a->density, a->jacobian, a->jacobian_u, a->jacobian_v,
                                                       a->jacobian_w, a->advection_dz, Um, Vm, Wm, Gc, DJR, Wp);
    // the column-march donor-cell pass of the handle path, one species at a
    // time through the one pass-1 field of the scratch
    const dim3 gu((unsigned)((g.nx + icar::upf::BX - 1) / icar::upf::BX),
                  (unsigned)((g.ny + icar::upf::BY - 1) / icar::upf::BY), 1u);
    for (int s = 0; s < a->n_species; s++) {
        icar::SpeciesPtrs sp{};
        sp.q0[0] = a->q_in[s];
        sp.q1[0] = q1;
        sp.out[0] = a->q_out[s];
        icar::k_mp_upwind_cols<<<gu, icar::upf::NT, icar::upf::SMEM, st>>>(g, sp, 1, 1, Um, Vm, Wm, Gc, DJR);
        icar::mp_corr_launch(st, 1, g, sp, 1, a->mpdata_fct ? 1 : 0, Um, Vm, Wp, Gc, DJR, a->advection_dz);
    }
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return fail(nullptr, ICAR_ADV_CUDA_ERROR, "launch failed: %s", cudaGetErrorString(ce));
    return ICAR_ADV_OK;
}
