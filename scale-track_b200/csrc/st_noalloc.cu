/*
 * st_noalloc.cu -- st_step_noalloc: one mixed-precision parcel step that allocates nothing.
 *
 * Some callers cannot call cudaMalloc: a host application that hands all device memory to
 * its own pool allocator, code running under a memory budget enforced by a framework, or a
 * plugin that must not grow the process's device footprint after set-up.  For them this
 * entry point runs the same step kernel as st_step on caller-owned parcel, fluid and source
 * arrays, and keeps its only scratch -- the fixed-point source accumulator and a control
 * block -- in a file-scope device array of fixed size.  It calls no cudaMalloc, cudaFree
 * or allocating library routine.
 *
 * The scratch array lives in every GPU that loads this library until the process exits.
 * Its device address is looked up once per device, on the first call made on that device
 * (cudaGetSymbolAddress with that device current), and kept for the life of the process: a
 * cudaDeviceReset of that device makes the kept address stale, so the entry point must not
 * be called on a device after it was reset.  Every call ends by reading the control block
 * back and synchronising the stream, so a call cannot be recorded into a CUDA graph: one
 * made on a capturing stream is rejected before anything is launched.  All calls share the
 * one array and it keeps the last call's contents: each call clears the accumulator and
 * control block it needs before use, and calls that overlap on the GPU (other streams or
 * host threads) race on the array.
 */
#include <climits>
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "scaletrack.h"
#include "st_internal.h"

using namespace st;

namespace {

constexpr int64_t NOALLOC_MAX_CELLS = ST_NOALLOC_MAX_CELLS;  /* include/scaletrack.h */
constexpr size_t ACC_BYTES = (size_t)NOALLOC_MAX_CELLS * 3 * sizeof(unsigned long long);
constexpr size_t HDR_BYTES = 512;  /* control block + cloud descriptor, padded */
static_assert(sizeof(CloudCtl) + sizeof(CloudK<double, float>) <= HDR_BYTES, "header");

/* [0, HDR_BYTES): CloudCtl, then CloudK<double,float>; [HDR_BYTES, ...): accumulator */
static __device__ __align__(256) unsigned char g_st_noalloc_scratch[HDR_BYTES + ACC_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
unsigned char* g_scratch_addr[MAX_DEVICES] = {nullptr};

int fail(int code, const char* msg)
{
    st_set_last_error(msg);
    return code;
}

/* Writes the control block and the cloud descriptor (passed by value: no host copy). */
__global__ void k_noalloc_init(CloudCtl ctl, CloudK<double, float> cloud, CloudCtl* ctl_dst,
                               CloudK<double, float>* cloud_dst)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        *ctl_dst = ctl;
        *cloud_dst = cloud;
    }
}

/* After the read-only probe: the scale maps the largest deposit of this call to 2^H. */
__global__ void k_noalloc_scale(CloudCtl* ctl)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        int em = ctl->emax;
        ctl->L = (em == EXP_NONE) ? -ctl->H : em - ctl->H;
        ctl->emax = EXP_NONE;
    }
}

/* Fixed point -> FP64 into the caller's [nCells][3] source (any length, scalar stores). */
__global__ void k_noalloc_finalize(const unsigned long long* __restrict__ acc,
                                   const CloudCtl* ctl, double* __restrict__ src,
                                   int64_t ncomp)
{
    const int L = ctl->L;
    const int k1 = L / 2, k2 = L - L / 2;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < ncomp;
         j += (int64_t)gridDim.x * blockDim.x) {
        const double v = (double)(long long)acc[j];
        src[j] = (v * __longlong_as_double((long long)(k1 + 1023) << 52)) *
                 __longlong_as_double((long long)(k2 + 1023) << 52);
    }
}

int quant_nbits(int64_t n_bound)
{
    int nb = 1;
    while (nb < 62 && ((int64_t)1 << nb) < n_bound) ++nb;
    return nb;
}

}  // namespace

extern "C" {

ST_API int64_t st_noalloc_max_cells(void) { return NOALLOC_MAX_CELLS; }

ST_API int st_step_noalloc(const st_params* p, const st_mesh_desc* m, int64_t n, double* x,
                           double* y, double* z, float* u, float* v, float* w, const float* d,
                           const float* U, double* source, double dt, double fluid_scale,
                           void* stream)
{
    if (!p || !m) return fail(ST_ERR_INVALID_ARGUMENT, "null params or mesh");
    if (p->precision != ST_PREC_MIXED || p->deposit != ST_DEPOSIT_DETERMINISTIC ||
        p->n_clouds != 1)
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "st_step_noalloc supports mixed precision, the deterministic deposit and "
                    "one cloud");
    if (p->drag_model != ST_DRAG_STOKES_IMPLICIT && p->drag_model != ST_DRAG_SCHILLER_NAUMANN)
        return fail(ST_ERR_INVALID_ARGUMENT, "unknown drag model");
    if (p->n_substeps < 1) return fail(ST_ERR_INVALID_ARGUMENT, "n_substeps must be >= 1");
    if (!(p->mu_c > 0) || !(p->rho_c > 0) || !(p->rho_d > 0))
        return fail(ST_ERR_INVALID_ARGUMENT, "mu_c, rho_c and rho_d must be positive");
    if (!(dt > 0) || !(dt < 1e300)) return fail(ST_ERR_INVALID_ARGUMENT, "dt must be positive");
    int64_t ncells = 1;
    for (int a = 0; a < 3; ++a) {
        if (m->n[a] < 1 || !(m->ending[a] > m->origin[a]))
            return fail(ST_ERR_INVALID_ARGUMENT, "bad mesh");
        ncells *= m->n[a];
    }
    if (ncells > NOALLOC_MAX_CELLS)
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "mesh too large for st_step_noalloc: at most st_noalloc_max_cells() "
                    "cells (the size of its fixed scratch array)");
    if (n < 0 || n > INT32_MAX) return fail(ST_ERR_INVALID_ARGUMENT, "parcel count out of range");
    if (n > 0 && (!x || !y || !z || !u || !v || !w || !d))
        return fail(ST_ERR_INVALID_ARGUMENT, "null parcel array");
    if (!U || !source) return fail(ST_ERR_INVALID_ARGUMENT, "null U or source");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
        return fail(ST_ERR_CUDA, "no current CUDA device");
    {
        /* the call synchronises the stream at its end, which a capture does not allow */
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const cudaError_t e = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cs);
        if (e != cudaSuccess) return fail(ST_ERR_CUDA, cudaGetErrorString(e));
        if (cs != cudaStreamCaptureStatusNone)
            return fail(ST_ERR_INVALID_ARGUMENT,
                        "st_step_noalloc synchronises its stream and cannot be captured into a "
                        "CUDA graph");
    }
    unsigned char* base;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_scratch_addr[dev]) {
            void* ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_st_noalloc_scratch);
            if (e != cudaSuccess || !ptr)
                return fail(ST_ERR_CUDA, cudaGetErrorString(e));
            g_scratch_addr[dev] = static_cast<unsigned char*>(ptr);
        }
        base = g_scratch_addr[dev];
    }
    CloudCtl* ctl = reinterpret_cast<CloudCtl*>(base);
    CloudK<double, float>* cloud =
        reinterpret_cast<CloudK<double, float>*>(base + sizeof(CloudCtl));
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(base + HDR_BYTES);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int64_t ncomp = ncells * 3;

    CloudCtl c0;
    std::memset(&c0, 0, sizeof c0);
    c0.emax = EXP_NONE;
    const int64_t bound = n * (int64_t)p->n_substeps > 2 ? n * (int64_t)p->n_substeps : 2;
    c0.H = 62 - QUANT_GROWTH_BITS - quant_nbits(bound);
    CloudK<double, float> ck;
    ck.x = x; ck.y = y; ck.z = z; ck.u = u; ck.v = v; ck.w = w; ck.d = d;
    ck.n = n;
    ck.tile0 = 0;
    ck.acc = acc;
    ck.src = nullptr;

    StepArgs<double, float> a;
    for (int k = 0; k < 3; ++k) {
        a.mesh.N[k] = m->n[k];
        a.mesh.origin[k] = m->origin[k];
        a.mesh.rD[k] = 1.0 / ((m->ending[k] - m->origin[k]) / (double)m->n[k]);
    }
    a.mesh.NxNy = m->n[0] * m->n[1];
    a.mesh.pad = 0;
    a.mesh.nCells = ncells;
    a.phys.mu = (float)p->mu_c;
    a.phys.rho_d = (float)p->rho_d;
    a.phys.rr = (float)(p->rho_d / p->rho_c);
    a.phys.nu = (float)(p->mu_c / p->rho_c);
    a.phys.rnu = (float)(p->rho_c / p->mu_c);
    a.phys.alpha = (float)p->drag_multiplier;
    a.phys.dscale = (float)p->diameter_scale;
    a.phys.drag = p->drag_model;
    a.phys.nsub = p->n_substeps;
    a.dtP = dt / (double)p->n_substeps;
    a.dtV = (float)a.dtP;
    split_fluid_scale<double, float>(fluid_scale, a.fscale, a.fscale_lo);
    a.nclouds = 1;
    a.U = U;
    a.clouds = cloud;
    a.ctl = ctl;
    a.total_tiles = (n + WARP_TILE - 1) / WARP_TILE;
    a.one = ck;

    cudaError_t e;
    if ((e = cudaMemsetAsync(acc, 0, (size_t)ncomp * sizeof(unsigned long long), s)) != cudaSuccess)
        return fail(ST_ERR_CUDA, cudaGetErrorString(e));
    k_noalloc_init<<<1, 32, 0, s>>>(c0, ck, ctl, cloud);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(ST_ERR_CUDA, cudaGetErrorString(e));
    if (n > 0) {
        int nsm = 148, occ = 1;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        occ = step_max_active_blocks<double, float>(DEP_DET1, 256);
        if (occ < 1) occ = 1;
        int64_t need = (a.total_tiles + 7) / 8;
        int grid = (int)(need < (int64_t)nsm * occ ? need : (int64_t)nsm * occ);
        if (grid < 1) grid = 1;
        if ((e = launch_step<double, float>(a, DEP_PROBE, grid, 256, s)) != cudaSuccess)
            return fail(ST_ERR_CUDA, cudaGetErrorString(e));
        k_noalloc_scale<<<1, 32, 0, s>>>(ctl);
        if ((e = launch_step<double, float>(a, DEP_DET1, grid, 256, s)) != cudaSuccess)
            return fail(ST_ERR_CUDA, cudaGetErrorString(e));
    }
    int fgrid = (int)((ncomp + 255) / 256 < 148 * 8 ? (ncomp + 255) / 256 : 148 * 8);
    k_noalloc_finalize<<<fgrid, 256, 0, s>>>(acc, ctl, source, ncomp);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail(ST_ERR_CUDA, cudaGetErrorString(e));

    CloudCtl out;
    if ((e = cudaMemcpyAsync(&out, ctl, sizeof out, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fail(ST_ERR_CUDA, cudaGetErrorString(e));
    if (out.lost) return fail(ST_ERR_PARCEL_OUTSIDE, "parcel(s) could not be located in the mesh");
    if (out.overflow)
        return fail(ST_ERR_SOURCE_RANGE, "deposit(s) exceeded the fixed-point range");
    return ST_OK;
}

}  // extern "C"
