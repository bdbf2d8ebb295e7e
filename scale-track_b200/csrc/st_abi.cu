/*
 * st_abi.cu -- the C ABI of libscaletrack.so (declared in include/scaletrack.h).
 *
 * Host side of the parcel step: handle and device memory management (cuboid and tet
 * meshes), the per-step launch sequence (probe -> step -> finalize, periodic re-sort), device
 * error reporting, CUDA-graph capture and the autotuner, the adjoint driver, device-side
 * initialisation and injection, restart files, and the shims with the reference's coupling
 * surface (allocate_array_ptr and evolve_cloud, A:1436-1528, in its synchronous and
 * asynchronous forms, with copied or mapped exchange arrays).  There is no CPU fallback:
 * without a CUDA device every entry point that needs one fails with ST_ERR_CUDA.
 *
 * Per-step launch sequence on the handle's stream (all clouds in each launch):
 *   [probe + set_scale]   only on the first step after st_set_parcels or a new dt
 *   [zero source]         only in ST_DEPOSIT_ATOMIC mode
 *   step                  k_step: the parcel step and the warp-aggregated deposit
 *   finalize              fixed point -> FP64 source and next scale; then a memset clears
 *                         the accumulators
 *   [sort]                every sort_interval steps
 */
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <climits>
#include <cmath>
#include <mutex>
#include <new>
#include <string>
#include <vector>
#include <map>
#include <algorithm>
#include <type_traits>

#include <cuda_runtime.h>

#include "scaletrack.h"
#include "st_internal.h"

using namespace st;

/* ------------------------------------------------------------------------------------ */
/* errors                                                                               */
/* ------------------------------------------------------------------------------------ */
static thread_local std::string g_err;

static int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

void st::st_set_last_error(const char* msg) { g_err = msg ? msg : ""; }

#define CK(...)                                                                             \
    do {                                                                                    \
        cudaError_t e_ = (__VA_ARGS__);                                                     \
        if (e_ != cudaSuccess)                                                              \
            return fail(ST_ERR_CUDA, "%s: %s (%s:%d)", #__VA_ARGS__, cudaGetErrorString(e_), \
                        __FILE__, __LINE__);                                                \
    } while (0)

/* ------------------------------------------------------------------------------------ */
/* the handle                                                                           */
/* ------------------------------------------------------------------------------------ */
struct CloudBufs {
    int64_t n = 0;
    int64_t shard_total = 0;   /* parcels of this cloud over all ranks of a sharded run */
    int64_t cap = 0;
    void* x[2] = {nullptr, nullptr};
    void* y[2] = {nullptr, nullptr};
    void* z[2] = {nullptr, nullptr};
    void* u[2] = {nullptr, nullptr};
    void* v[2] = {nullptr, nullptr};
    void* w[2] = {nullptr, nullptr};
    void* d[2] = {nullptr, nullptr};
    int32_t* id[2] = {nullptr, nullptr};
    int32_t* cell[2] = {nullptr, nullptr};  /* owning tet (tet meshes) */
    uint32_t* keys[2] = {nullptr, nullptr};
    uint32_t* perm[2] = {nullptr, nullptr};
    int cur = 0;
};

struct ProfRec {
    int kind;
    cudaEvent_t a, b;
};

/* Device memory of the mean-source adjoint: checkpoints of the last forward pass, the
 * records of one segment, the cotangent and the per-block parameter partials. */
struct AdjTape {
    bool valid = false;
    int cloud = -1;
    int T = 0, C = 0, nseg = 0, grid = 0, limbs = 1;
    int64_t n = 0;
    double dt = 0.0;
    std::vector<double> fs;     /* host copy of the per-step factors of the forward pass */
    size_t bytes = 0;
    void* mem = nullptr;        /* one allocation, carved below */
    void* ck_x = nullptr;
    void* ck_v = nullptr;
    void* rec_v = nullptr;
    int32_t* rec_c = nullptr;
    uint8_t* rec_b = nullptr;
    double* G = nullptr;
    void* adj_v = nullptr;
    double* partials = nullptr;
    void* fsd = nullptr;
    double* mean = nullptr;
    CloudCtl* ctl = nullptr;
    unsigned long long* acc = nullptr;
};

struct st_handle {
    st_params p;
    st_mesh_desc m;
    int device = 0;
    int nsm = 148;         /* streaming multiprocessors of the device */
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int dep = DEP_DET1;
    int limbs = 1;
    int64_t ncells = 0;
    int64_t stride = 0;   /* per-cloud component stride of source/accumulator arrays */
    size_t psz = 4, vsz = 4;
    void* dU = nullptr;
    double* dsrc = nullptr;
    unsigned long long* dacc = nullptr;
    CloudCtl* dctl = nullptr;
    unsigned int* dcounter = nullptr;
    unsigned long long* dcount = nullptr;  /* scratch counter (outside parcels) */
    void* dclouds = nullptr;
    std::vector<unsigned char> hclouds;      /* host image of the CloudK array */
    std::vector<unsigned char> hclouds2;     /* host image of the two-parity pair (capture) */
    std::vector<CloudBufs> clouds;
    bool clouds_dirty = true;
    bool need_probe = true;
    double last_dt = 0.0;
    int64_t steps = 0;
    int steps_since_sort = 0;
    int block = 256;
    int grid = 0;
    bool ring = true;      /* ST_STEP_KERNEL_RING for single-cloud steps */
    int32_t* dexp = nullptr;   /* [nclouds] largest-deposit exponents of a sharded step */
    float* dsrc32 = nullptr;   /* when set, the finalize also writes the FP32 source here
                                  ([nclouds][stride]; the coupling's 4-byte exchange) */
    /* Overlapped finalize (one cloud, deterministic deposit, outside graph capture and the
     * sharded phases): step n deposits into accumulator par, k_next_scale keeps its scale in
     * dLfin[par] and sets the next one, and the finalize and clearing of accumulator par run
     * on fin_stream while step n + 1 runs on the handle's stream with the other accumulator. */
    bool fin_overlap = true;
    int64_t wait_cycles = 0;     /* ring kernels' pipeline-wait limit (st_set_wait_limit),
                                    negated for the stall test */
    cudaStream_t fin_stream = nullptr;
    cudaEvent_t ev_step[2] = {nullptr, nullptr};
    cudaEvent_t ev_fin[2] = {nullptr, nullptr};
    bool fin_pending[2] = {false, false};
    int par = 0;
    unsigned long long* dacc2 = nullptr;
    int32_t* dLfin = nullptr;  /* [2][nclouds] */
    bool shard_probed = false; /* st_shard_probe ran; its exponents are in dexp */
    int key_bits = 24;     /* bits of the sort key, at most COUNT_SORT_MAX_BITS */
    int key_shift = 0;     /* low bits dropped to fit them (sort keys are for locality only) */
    bool morton = true;
    int64_t total_tiles = 0;
    int64_t launches = 0;
    bool prof = false;
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> pool;
    int64_t prof_launches[ST_KERNEL_KINDS] = {};
    double prof_ms[ST_KERNEL_KINDS] = {};
    void* dstage = nullptr;
    size_t stage_bytes = 0;
    /* counting-sort bins shared by the clouds (key ranges up to 2^COUNT_SORT_MAX_BITS) */
    uint32_t* dbins = nullptr;
    uint32_t* doffs = nullptr;
    void* dscan = nullptr;
    size_t scan_bytes = 0;
    AdjTape adj;
    /* unstructured tetrahedral mesh */
    bool tet = false;
    TetMeshK tmesh = {};
    double* d_verts = nullptr;
    int32_t* d_tets = nullptr;
    double4* d_planes = nullptr;            /* [nt][4] face planes */
    float4* d_planes32 = nullptr;           /* [nt][4] the same in FP32 */
    int32_t* d_nbr = nullptr;
    unsigned long long* d_hops = nullptr;   /* walk-length histogram [8] */
    /* CUDA-graph replay of a step sequence */
    bool capturing = false;
    int cap_parity = 0;          /* which of the two descriptor arrays the captured step uses */
    void* dclouds2 = nullptr;    /* descriptors for the current and the re-sorted buffers */
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int graph_steps = 0;
    int64_t graph_launches = 0;
};

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int now = -1;
        if (prev >= 0 && cudaGetDevice(&now) == cudaSuccess && now != prev) cudaSetDevice(prev);
    }
};

template <class P>
MeshK<P> mesh_k(const st_handle* h)
{
    MeshK<P> k;
    for (int a = 0; a < 3; ++a) {
        k.N[a] = h->m.n[a];
        k.origin[a] = (P)h->m.origin[a];
        double L = h->m.ending[a] - h->m.origin[a];
        double D = L / (double)h->m.n[a];
        k.rD[a] = (P)(1.0 / D);
    }
    k.NxNy = h->m.n[0] * h->m.n[1];
    k.pad = 0;
    k.nCells = h->ncells;
    return k;
}

template <class V>
PhysK<V> phys_k(const st_handle* h)
{
    PhysK<V> k;
    k.mu = (V)h->p.mu_c;
    k.rho_d = (V)h->p.rho_d;
    k.rr = (V)(h->p.rho_d / h->p.rho_c);
    k.nu = (V)(h->p.mu_c / h->p.rho_c);
    k.rnu = (V)(h->p.rho_c / h->p.mu_c);
    k.alpha = (V)h->p.drag_multiplier;
    k.dscale = (V)h->p.diameter_scale;
    k.drag = h->p.drag_model;
    k.nsub = h->p.n_substeps;
    return k;
}

int quant_nbits(int64_t n_bound)
{
    int nb = 1;
    while (nb < 62 && ((int64_t)1 << nb) < n_bound) ++nb;
    return nb;
}

cudaEvent_t take_event(st_handle* h)
{
    if (!h->pool.empty()) {
        cudaEvent_t e = h->pool.back();
        h->pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}

/* Brackets one kernel launch with events when profiling is on. */
struct ProfScope {
    st_handle* h;
    int kind;
    cudaStream_t s;
    cudaEvent_t a = nullptr;
    ProfScope(st_handle* hh, int k, cudaStream_t st = nullptr)
        : h(hh), kind(k), s(st ? st : hh->stream)
    {
        if (h->prof) {
            a = take_event(h);
            if (a && cudaEventRecord(a, s) != cudaSuccess) {
                cudaGetLastError();
                h->pool.push_back(a);
                a = nullptr;
            }
        }
    }
    ~ProfScope()
    {
        /* a launch whose events could not be recorded is left out of the profile */
        if (h->prof && a) {
            cudaEvent_t b = take_event(h);
            if (b && cudaEventRecord(b, s) == cudaSuccess) {
                h->recs.push_back({kind, a, b});
                return;
            }
            cudaGetLastError();
            h->pool.push_back(a);
            if (b) h->pool.push_back(b);
        }
    }
};

/* Blocks per cloud of the finalize pass: four 256-thread blocks per SM over all clouds
 * (measured at 128^3 cells: 23 us against 28 us with eight), each thread looping over
 * groups of four components. */
int finalize_grid(const st_handle* h)
{
    int64_t gx = (h->stride / COMP_ALIGN + 255) / 256;
    const int64_t cap = ((int64_t)h->nsm * 4 + h->p.n_clouds - 1) / h->p.n_clouds;
    if (gx > cap) gx = cap;
    if (gx < 1) gx = 1;
    return (int)gx;
}

/* Orders the handle's stream after every finalize still pending on fin_stream: the source
 * and both accumulators are then final on the handle's stream. */
int join_fin(st_handle* h)
{
    for (int p = 0; p < 2; ++p)
        if (h->fin_pending[p]) {
            CK(cudaStreamWaitEvent(h->stream, h->ev_fin[p], 0));
            h->fin_pending[p] = false;
        }
    return ST_OK;
}

/* Waits on the host for the finalize stream (before the handle's stream changes, a graph is
 * captured or the handle goes away). */
int drain_fin(st_handle* h)
{
    if (h->fin_stream) CK(cudaStreamSynchronize(h->fin_stream));
    h->fin_pending[0] = h->fin_pending[1] = false;
    return ST_OK;
}

/* The second accumulator, scale slots, stream and events of the overlapped finalize, made on
 * the first overlapped step. */
int ensure_overlap(st_handle* h)
{
    if (h->fin_stream) return ST_OK;
    const size_t bytes = (size_t)h->stride * h->p.n_clouds * h->limbs * 8;
    if (!h->dacc2) {
        CK(cudaMalloc((void**)&h->dacc2, bytes));
        CK(cudaMemsetAsync(h->dacc2, 0, bytes, h->stream));
    }
    if (!h->dLfin) CK(cudaMalloc((void**)&h->dLfin, 2 * sizeof(int32_t) * h->p.n_clouds));
    for (int p = 0; p < 2; ++p) {
        if (!h->ev_step[p]) CK(cudaEventCreateWithFlags(&h->ev_step[p], cudaEventDisableTiming));
        if (!h->ev_fin[p]) CK(cudaEventCreateWithFlags(&h->ev_fin[p], cudaEventDisableTiming));
    }
    CK(cudaStreamCreateWithFlags(&h->fin_stream, cudaStreamNonBlocking));
    return ST_OK;
}

int ensure_stage(st_handle* h, size_t bytes)
{
    if (h->stage_bytes >= bytes) return ST_OK;
    if (h->dstage) cudaFree(h->dstage);
    h->dstage = nullptr;
    h->stage_bytes = 0;
    CK(cudaMalloc(&h->dstage, bytes));
    h->stage_bytes = bytes;
    return ST_OK;
}

/* Reads the control blocks; reports (and clears) lost parcels and range errors. */
int check_device_errors(st_handle* h)
{
    const int nc = h->p.n_clouds;
    std::vector<CloudCtl> ctl(nc);
    CK(cudaMemcpyAsync(ctl.data(), h->dctl, sizeof(CloudCtl) * nc, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    unsigned long long lost = 0, ovf = 0;
    int fault = 0;
    for (int c = 0; c < nc; ++c) {
        lost += ctl[c].lost;
        ovf += ctl[c].overflow;
        fault |= ctl[c].fault;
    }
    if (lost || ovf || fault) {
        for (int c = 0; c < nc; ++c) ctl[c].lost = ctl[c].overflow = ctl[c].fault = 0;
        CK(cudaMemcpyAsync(h->dctl, ctl.data(), sizeof(CloudCtl) * nc, cudaMemcpyHostToDevice,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (fault)
            return fail(ST_ERR_CUDA,
                        "a step kernel gave up waiting on its shared-memory pipeline (fault "
                        "bits %d); that step's results are incomplete", fault);
        /* lost parcels take precedence in the status; the message counts both */
        if (lost)
            return fail(ST_ERR_PARCEL_OUTSIDE,
                        "%llu parcel(s) could not be located in the mesh and were left "
                        "unchanged; %llu deposit component(s) out of range", lost, ovf);
        return fail(ST_ERR_SOURCE_RANGE,
                    "%llu deposit component(s) were non-finite or exceeded the fixed-point "
                    "range of the deterministic source and were dropped", ovf);
    }
    return ST_OK;
}

template <class P, class V>
SortBufs<P, V> sort_bufs(const st_handle* h, CloudBufs& c)
{
    SortBufs<P, V> b;
    b.bins = h->dbins;
    b.offsets = h->doffs;
    b.scan_temp = h->dscan;
    b.scan_temp_bytes = h->scan_bytes;
    for (int k = 0; k < 2; ++k) {
        b.x[k] = (P*)c.x[k];
        b.y[k] = (P*)c.y[k];
        b.z[k] = (P*)c.z[k];
        b.u[k] = (V*)c.u[k];
        b.v[k] = (V*)c.v[k];
        b.w[k] = (V*)c.w[k];
        b.d[k] = (V*)c.d[k];
        b.id[k] = c.id[k];
        b.cell[k] = c.cell[k];
        b.keys[k] = c.keys[k];
        b.perm[k] = c.perm[k];
    }
    return b;
}

template <class P, class V>
int upload_clouds(st_handle* h)
{
    const int nc = h->p.n_clouds;
    std::vector<CloudK<P, V>> v(nc);
    int64_t tiles = 0;
    for (int c = 0; c < nc; ++c) {
        CloudBufs& b = h->clouds[c];
        CloudK<P, V>& k = v[c];
        k.x = (P*)b.x[b.cur];
        k.y = (P*)b.y[b.cur];
        k.z = (P*)b.z[b.cur];
        k.u = (V*)b.u[b.cur];
        k.v = (V*)b.v[b.cur];
        k.w = (V*)b.w[b.cur];
        k.d = (const V*)b.d[b.cur];
        k.n = b.n;
        k.tile0 = tiles;
        k.acc = h->dacc + (int64_t)c * h->stride * h->limbs;
        k.src = h->dsrc + (int64_t)c * h->stride;
        k.cell = b.cell[b.cur];
        tiles += (b.n + WARP_TILE - 1) / WARP_TILE;
    }
    h->total_tiles = tiles;
    h->hclouds.resize(sizeof(CloudK<P, V>) * nc);
    memcpy(h->hclouds.data(), v.data(), h->hclouds.size());
    CK(cudaMemcpyAsync(h->dclouds, h->hclouds.data(), h->hclouds.size(), cudaMemcpyHostToDevice,
                       h->stream));
    h->clouds_dirty = false;
    return ST_OK;
}

template <class P, class V>
int do_sort_all(st_handle* h)
{
    const MeshK<P> mk = mesh_k<P>(h);
    for (auto& c : h->clouds) {
        if (c.n <= 1) continue;
        SortBufs<P, V> b = sort_bufs<P, V>(h, c);
        int nl = 0;
        {
            ProfScope ps(h, ST_KERNEL_SORT);
            CK(sort_cloud<P, V>(b, c.cur, c.n, mk, h->key_bits, h->key_shift, h->morton, h->stream,
                                &nl));
        }
        h->launches += nl;
        c.cur = 1 - c.cur;
    }
    h->clouds_dirty = true;
    h->steps_since_sort = 0;
    if (h->capturing) h->cap_parity ^= 1;
    return ST_OK;
}

/* Phases of one step.  PH_ALL is st_step.  A sharded step (one handle per rank, parcels
 * split over the ranks) runs PH_PROBE (first step only), PH_DEPOSIT and PH_FINISH as separate
 * calls, and the caller combines the ranks' exponents (max) and accumulators (sum) between
 * them; the exponents travel through the contiguous buffer h->dexp. */
enum StepPhase { PH_ALL = 0, PH_PROBE = 1, PH_DEPOSIT = 2, PH_FINISH = 3 };

/* The launch sequence shared by hex and tet meshes: `launch(dep)` launches the step kernel
 * of the mesh with deposit mode dep (DEP_PROBE for the read-only pass), `sort()` re-sorts
 * every cloud. */
template <class L, class S>
int step_phases(st_handle* h, double dt, int phase, bool empty, L&& launch, S&& sort,
                unsigned long long* acc_ovl = nullptr)
{
    const bool det = (h->dep == DEP_DET1 || h->dep == DEP_DET2);
    const int nc = h->p.n_clouds;
    if (phase != PH_ALL && !det)
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "sharded steps need the deterministic deposit (integer accumulators)");
    if (phase == PH_ALL && empty) return ST_OK;
    if (phase == PH_PROBE) {
        if (!empty) {
            ProfScope ps(h, ST_KERNEL_PROBE);
            CK(launch(DEP_PROBE));
            h->launches += 1;
        }
        CK(launch_ctl_exponents(h->dctl, h->dexp, nc, false, h->stream));
        h->shard_probed = true;
        h->last_dt = dt;
        return ST_OK;
    }
    if (phase != PH_FINISH) {
        if (det && phase == PH_DEPOSIT && h->shard_probed) {
            /* the first-step scale from the exponents every rank agreed on */
            CK(launch_ctl_exponents(h->dctl, h->dexp, nc, true, h->stream));
            CK(launch_set_scale(h->dctl, nc, h->stream));
            h->launches += 1;
            h->shard_probed = false;
            h->need_probe = false;
        } else if (det && (h->need_probe || dt != h->last_dt)) {
            if (phase == PH_DEPOSIT)
                return fail(ST_ERR_INVALID_ARGUMENT,
                            "st_shard_probe must precede the first sharded step (and a new dt)");
            {
                ProfScope ps(h, ST_KERNEL_PROBE);
                CK(launch(DEP_PROBE));
            }
            {
                ProfScope ps(h, ST_KERNEL_OTHER);
                CK(launch_set_scale(h->dctl, nc, h->stream));
            }
            h->launches += 2;
            h->need_probe = false;
        }
        h->last_dt = dt;
        if (!det) {
            ProfScope ps(h, ST_KERNEL_OTHER);
            CK(launch_zero_f64(h->dsrc, (int64_t)nc * h->stride, h->stream));
            h->launches += 1;
        }
        if (!empty) {
            ProfScope ps(h, ST_KERNEL_STEP);
            CK(launch(h->dep));
            h->launches += 1;
        }
        if (phase == PH_DEPOSIT) {
            CK(launch_ctl_exponents(h->dctl, h->dexp, nc, false, h->stream));
            return ST_OK;
        }
    }
    if (det && acc_ovl) {
        /* overlapped finalize: the next scale now, in stream order; the conversion and the
         * clearing of this step's accumulator on fin_stream, concurrent with the next step */
        const int p = h->par;
        int32_t* Lf = h->dLfin + (size_t)p * nc;
        CK(launch_next_scale(h->dctl, Lf, nc, h->stream));
        CK(cudaEventRecord(h->ev_step[p], h->stream));
        CK(cudaStreamWaitEvent(h->fin_stream, h->ev_step[p], 0));
        {
            ProfScope ps(h, ST_KERNEL_FINALIZE, h->fin_stream);
            CK(launch_finalize(h->limbs, acc_ovl, h->dsrc, h->dsrc32, h->dctl, Lf, h->dcounter,
                               nc, h->stride, finalize_grid(h), h->fin_stream));
        }
        CK(cudaMemsetAsync(acc_ovl, 0, (size_t)h->stride * nc * h->limbs * 8, h->fin_stream));
        CK(cudaEventRecord(h->ev_fin[p], h->fin_stream));
        h->fin_pending[p] = true;
        h->par ^= 1;
        h->launches += 2;
    } else if (det) {
        if (phase == PH_FINISH) CK(launch_ctl_exponents(h->dctl, h->dexp, nc, true, h->stream));
        {
            ProfScope ps(h, ST_KERNEL_FINALIZE);
            CK(launch_finalize(h->limbs, h->dacc, h->dsrc, h->dsrc32, h->dctl, nullptr,
                               h->dcounter, nc, h->stride, finalize_grid(h), h->stream));
            h->launches += 1;
        }
        CK(cudaMemsetAsync(h->dacc, 0, (size_t)h->stride * nc * h->limbs * 8, h->stream));
    }
    h->steps += 1;
    h->steps_since_sort += 1;
    if (h->p.sort_interval > 0 && h->steps_since_sort >= h->p.sort_interval) return sort();
    return ST_OK;
}

template <class V>
int do_step_tet(st_handle* h, double dt, double fscale, int phase);

template <class P, class V>
int do_step(st_handle* h, double dt, double fscale, int phase = PH_ALL)
{
    int rc;
    if constexpr (std::is_same<P, double>::value) {
        if (h->tet) return do_step_tet<V>(h, dt, fscale, phase);
    }
    if (!h->capturing && h->clouds_dirty && (rc = upload_clouds<P, V>(h)) != ST_OK) return rc;
    const bool ovl = h->fin_overlap && phase == PH_ALL && !h->capturing &&
                     (h->dep == DEP_DET1 || h->dep == DEP_DET2) && h->p.n_clouds == 1;
    if ((rc = ovl ? ensure_overlap(h) : join_fin(h))) return rc;
    StepArgs<P, V> a;
    a.mesh = mesh_k<P>(h);
    a.phys = phys_k<V>(h);
    a.dtP = (P)dt / (P)h->p.n_substeps;
    a.dtV = (V)a.dtP;
    split_fluid_scale<P, V>(fscale, a.fscale, a.fscale_lo);
    a.nclouds = h->p.n_clouds;
    a.U = (const V*)h->dU;
    a.clouds = h->capturing
                   ? (const CloudK<P, V>*)h->dclouds2 + (size_t)h->cap_parity * h->p.n_clouds
                   : (const CloudK<P, V>*)h->dclouds;
    a.ctl = h->dctl;
    a.total_tiles = h->total_tiles;
    a.wait_cycles = h->wait_cycles;
    if (h->p.n_clouds == 1) {
        const std::vector<unsigned char>& hc = h->capturing ? h->hclouds2 : h->hclouds;
        const size_t off = h->capturing ? (size_t)h->cap_parity * sizeof(CloudK<P, V>) : 0;
        memcpy(&a.one, hc.data() + off, sizeof(CloudK<P, V>));
    } else {
        memset(&a.one, 0, sizeof a.one);
    }
    unsigned long long* acc_ovl = nullptr;
    if (ovl) {
        /* this step deposits into accumulator par, cleared by the finalize two steps back */
        acc_ovl = h->par ? h->dacc2 : h->dacc;
        a.one.acc = acc_ovl;
        if (h->fin_pending[h->par]) {
            CK(cudaStreamWaitEvent(h->stream, h->ev_fin[h->par], 0));
            h->fin_pending[h->par] = false;
        }
    }
    int grid = h->grid;
    const int64_t warps_per_block = h->block / 32;
    const int64_t need = (a.total_tiles + warps_per_block - 1) / warps_per_block;
    if (grid > need) grid = (int)need;
    if (grid < 1) grid = 1;
    auto launch = [&](int dep) -> cudaError_t {
        if (dep != DEP_PROBE && h->ring && ring_eligible<P, V>(a, dep))
            return launch_step_ring<P, V>(a, dep, h->nsm, h->stream);
        return launch_step<P, V>(a, dep, grid, h->block, h->stream);
    };
    return step_phases(h, dt, phase, a.total_tiles == 0, launch,
                       [&] { return do_sort_all<P, V>(h); }, acc_ovl);
}

/* The step on a tetrahedral mesh: the launch sequence of do_step with the face-walk kernel
 * (st_tet.cu). */
template <class V>
int do_step_tet(st_handle* h, double dt, double fscale, int phase)
{
    int rc;
    if ((rc = join_fin(h))) return rc;
    if (!h->capturing && h->clouds_dirty && (rc = upload_clouds<double, V>(h)) != ST_OK) return rc;
    TetStepArgs<V> a;
    a.mesh = h->tmesh;
    a.phys = phys_k<V>(h);
    a.dtP = dt / (double)h->p.n_substeps;
    a.dtV = (V)a.dtP;
    split_fluid_scale<double, V>(fscale, a.fscale, a.fscale_lo);
    a.nclouds = h->p.n_clouds;
    a.U = (const V*)h->dU;
    a.clouds = h->capturing
                   ? (const CloudK<double, V>*)h->dclouds2 + (size_t)h->cap_parity * h->p.n_clouds
                   : (const CloudK<double, V>*)h->dclouds;
    a.ctl = h->dctl;
    a.total_tiles = h->total_tiles;
    a.wait_cycles = h->wait_cycles;
    a.hop_hist = h->d_hops;
    if (h->p.n_clouds == 1) {
        const std::vector<unsigned char>& hc = h->capturing ? h->hclouds2 : h->hclouds;
        const size_t off = h->capturing ? (size_t)h->cap_parity * sizeof(CloudK<double, V>) : 0;
        memcpy(&a.one, hc.data() + off, sizeof(CloudK<double, V>));
    } else {
        memset(&a.one, 0, sizeof a.one);
    }
    int grid = h->grid;
    const int64_t need = (a.total_tiles + h->block / 32 - 1) / (h->block / 32);
    if (grid > need) grid = (int)need;
    if (grid < 1) grid = 1;
    auto launch = [&](int dep) -> cudaError_t {
        if (dep != DEP_PROBE && h->ring && tet_ring_eligible<V>(a, dep))
            return launch_step_tet_ring<V>(a, dep, h->nsm, h->stream);
        return launch_step_tet<V>(a, dep, grid, h->block, h->stream);
    };
    return step_phases(h, dt, phase, a.total_tiles == 0, launch,
                       [&] { return do_sort_all<double, V>(h); });
}

/* Parcels generated on the device instead of uploaded (st_init_parcels). */
struct InitSpec {
    uint64_t seed;
    double d_min, d_max;
};

template <class P, class V>
int do_set_parcels(st_handle* h, int cloud, int64_t n, const double* xyz, const double* uvw,
                   const double* d, const int32_t* hint, const InitSpec* gen = nullptr)
{
    CloudBufs& c = h->clouds[cloud];
    if (n > c.cap) {
        /* a failed allocation below leaves an empty cloud that the next call reallocates */
        c.cap = 0;
        c.n = 0;
        h->clouds_dirty = true;
        for (int k = 0; k < 2; ++k) {
            void** arrs[] = {&c.x[k], &c.y[k], &c.z[k], &c.u[k], &c.v[k], &c.w[k], &c.d[k]};
            for (int a = 0; a < 7; ++a) {
                if (*arrs[a]) cudaFree(*arrs[a]);
                *arrs[a] = nullptr;
                CK(cudaMalloc(arrs[a], (size_t)n * (a < 3 ? sizeof(P) : sizeof(V))));
            }
            if (c.id[k]) cudaFree(c.id[k]);
            if (c.keys[k]) cudaFree(c.keys[k]);
            if (c.perm[k]) cudaFree(c.perm[k]);
            if (c.cell[k]) cudaFree(c.cell[k]);
            c.id[k] = nullptr;
            c.cell[k] = nullptr;
            c.keys[k] = c.perm[k] = nullptr;
            if (h->tet) CK(cudaMalloc(&c.cell[k], (size_t)n * sizeof(int32_t)));
            CK(cudaMalloc(&c.id[k], (size_t)n * sizeof(int32_t)));
            CK(cudaMalloc(&c.keys[k], (size_t)n * sizeof(uint32_t)));
            CK(cudaMalloc(&c.perm[k], (size_t)n * sizeof(uint32_t)));
        }
        c.cap = n;
    }
    c.n = n;
    c.cur = 0;
    if (n > 0 && gen) {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(launch_init_cloud<P, V>(gen->seed, cloud, h->p.n_clouds, n, mesh_k<P>(h), h->m.origin,
                                   h->m.ending, gen->d_min, gen->d_max, (P*)c.x[0],
                                   (P*)c.y[0], (P*)c.z[0], (V*)c.u[0], (V*)c.v[0], (V*)c.w[0],
                                   (V*)c.d[0], c.id[0], h->stream));
        h->launches += 1;
    }
    if (n > 0 && !gen) {
        std::vector<P> hp(n);
        std::vector<V> hv(n);
        std::vector<int32_t> hid(n);
        for (int a = 0; a < 3; ++a) {
            for (int64_t i = 0; i < n; ++i) hp[i] = (P)xyz[a * n + i];
            void* dst = a == 0 ? c.x[0] : (a == 1 ? c.y[0] : c.z[0]);
            CK(cudaMemcpyAsync(dst, hp.data(), n * sizeof(P), cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));   /* hp is reused */
        }
        for (int a = 0; a < 4; ++a) {
            const double* srcp = a < 3 ? uvw + a * n : d;
            for (int64_t i = 0; i < n; ++i) hv[i] = (V)srcp[i];
            void* dst = a == 0 ? c.u[0] : (a == 1 ? c.v[0] : (a == 2 ? c.w[0] : c.d[0]));
            CK(cudaMemcpyAsync(dst, hv.data(), n * sizeof(V), cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));   /* hv is reused */
        }
        for (int64_t i = 0; i < n; ++i) hid[i] = (int32_t)i;
        /* every upload is ordered on the handle's stream: a plain cudaMemcpy runs on the
         * legacy stream, which the handle's non-blocking stream does not wait for */
        CK(cudaMemcpyAsync(c.id[0], hid.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));   /* hid is freed at the end of this block */
    }
    if (n > 0) {
        /* every parcel must start inside the mesh: the reference would index out of bounds */
        CK(cudaMemsetAsync(h->dcount, 0, sizeof(unsigned long long), h->stream));
        if (h->tet) {
            /* walk from the caller's hint to the owning tet */
            CK(cudaMemcpyAsync(c.cell[1], hint, n * sizeof(int32_t), cudaMemcpyHostToDevice,
                               h->stream));
            ProfScope ps(h, ST_KERNEL_OTHER);
            TetMeshK lm = h->tmesh;
            lm.hop_limit = 1 << 20;   /* bounded: a walk that cycles counts as outside */
            CK(launch_tet_locate(lm, (const double*)c.x[0], (const double*)c.y[0],
                                 (const double*)c.z[0], c.cell[1], n, c.cell[0], h->dcount,
                                 h->stream));
            h->launches += 1;
        } else {
            ProfScope ps(h, ST_KERNEL_OTHER);
            CK(cells_cloud<P>((const P*)c.x[0], (const P*)c.y[0], (const P*)c.z[0], nullptr, n,
                              mesh_k<P>(h), (int32_t*)c.keys[0], h->dcount, h->stream));
            h->launches += 1;
        }
        unsigned long long outside = 0;
        CK(cudaMemcpyAsync(&outside, h->dcount, sizeof outside, cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (outside) {
            c.n = 0;
            h->clouds_dirty = true;
            return fail(ST_ERR_PARCEL_OUTSIDE,
                        "%llu of %lld parcels of cloud %d lie outside the mesh", outside,
                        (long long)n, cloud);
        }
    }
    h->clouds_dirty = true;
    h->need_probe = true;
    if (h->p.sort_interval > 0 && n > 1) {
        CloudBufs& cc = h->clouds[cloud];
        SortBufs<P, V> b = sort_bufs<P, V>(h, cc);
        int nl = 0;
        ProfScope ps(h, ST_KERNEL_SORT);
        CK(sort_cloud<P, V>(b, cc.cur, cc.n, mesh_k<P>(h), h->key_bits, h->key_shift, h->morton,
                            h->stream, &nl));
        h->launches += nl;
        cc.cur = 1 - cc.cur;
    }
    return ST_OK;
}

/* Appends m parcels to a cloud in place (injection): the buffers grow by at least half when
 * full (the current parcels are copied on the device), the new parcels go to the end of the
 * current buffers with ids n .. n+m-1, and the next step re-derives the fixed-point scale. */
template <class P, class V>
int do_append_parcels(st_handle* h, int cloud, int64_t m, const double* xyz, const double* uvw,
                      const double* d)
{
    CloudBufs& c = h->clouds[cloud];
    const int64_t n = c.n, nn = n + m;
    if (nn > c.cap) {
        int64_t cap = c.cap + c.cap / 2;
        if (cap < nn) cap = nn;
        /* every new buffer is allocated before anything is replaced, so a failure leaves the
         * cloud as it was */
        void** arrs[2][8] = {{&c.x[0], &c.y[0], &c.z[0], &c.u[0], &c.v[0], &c.w[0], &c.d[0],
                              (void**)&c.id[0]},
                             {&c.x[1], &c.y[1], &c.z[1], &c.u[1], &c.v[1], &c.w[1], &c.d[1],
                              (void**)&c.id[1]}};
        size_t es[8];
        for (int a = 0; a < 8; ++a)
            es[a] = a < 3 ? sizeof(P) : (a < 7 ? sizeof(V) : sizeof(int32_t));
        std::vector<void*> fresh;
        auto grab = [&](size_t bytes) -> void* {
            void* p = nullptr;
            if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
            fresh.push_back(p);
            return p;
        };
        void* nb[2][8];
        void* nkeys[2];
        void* nperm[2];
        bool ok = true;
        for (int k = 0; k < 2 && ok; ++k) {
            for (int a = 0; a < 8 && ok; ++a) ok = (nb[k][a] = grab((size_t)cap * es[a])) != nullptr;
            ok = ok && (nkeys[k] = grab((size_t)cap * sizeof(uint32_t))) != nullptr;
            ok = ok && (nperm[k] = grab((size_t)cap * sizeof(uint32_t))) != nullptr;
        }
        if (!ok) {
            for (void* p : fresh) cudaFree(p);
            cudaGetLastError();
            return fail(ST_ERR_OUT_OF_MEMORY, "no device memory for %lld parcels", (long long)cap);
        }
        for (int a = 0; a < 8 && n > 0; ++a)
            CK(cudaMemcpyAsync(nb[0][a], *arrs[c.cur][a], (size_t)n * es[a],
                               cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int k = 0; k < 2; ++k) {
            for (int a = 0; a < 8; ++a) {
                if (*arrs[k][a]) cudaFree(*arrs[k][a]);
                *arrs[k][a] = nb[k][a];
            }
            if (c.keys[k]) cudaFree(c.keys[k]);
            if (c.perm[k]) cudaFree(c.perm[k]);
            c.keys[k] = (uint32_t*)nkeys[k];
            c.perm[k] = (uint32_t*)nperm[k];
        }
        c.cap = cap;
        c.cur = 0;
        h->clouds_dirty = true;
    }
    const int k = c.cur;
    std::vector<P> hp(m);
    std::vector<V> hv(m);
    std::vector<int32_t> hid(m);
    P* dstp[3] = {(P*)c.x[k] + n, (P*)c.y[k] + n, (P*)c.z[k] + n};
    for (int a = 0; a < 3; ++a) {
        for (int64_t i = 0; i < m; ++i) hp[i] = (P)xyz[a * m + i];
        CK(cudaMemcpyAsync(dstp[a], hp.data(), m * sizeof(P), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    V* dstv[4] = {(V*)c.u[k] + n, (V*)c.v[k] + n, (V*)c.w[k] + n, (V*)c.d[k] + n};
    for (int a = 0; a < 4; ++a) {
        const double* srcp = a < 3 ? uvw + a * m : d;
        for (int64_t i = 0; i < m; ++i) hv[i] = (V)srcp[i];
        CK(cudaMemcpyAsync(dstv[a], hv.data(), m * sizeof(V), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    for (int64_t i = 0; i < m; ++i) hid[i] = (int32_t)(n + i);
    CK(cudaMemcpyAsync(c.id[k] + n, hid.data(), m * sizeof(int32_t), cudaMemcpyHostToDevice,
                       h->stream));
    /* the new parcels must lie inside the mesh */
    CK(cudaMemsetAsync(h->dcount, 0, sizeof(unsigned long long), h->stream));
    {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(cells_cloud<P>(dstp[0], dstp[1], dstp[2], nullptr, m, mesh_k<P>(h),
                          (int32_t*)c.keys[0], h->dcount, h->stream));
        h->launches += 1;
    }
    unsigned long long outside = 0;
    CK(cudaMemcpyAsync(&outside, h->dcount, sizeof outside, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (outside)
        return fail(ST_ERR_PARCEL_OUTSIDE, "%llu of %lld appended parcels lie outside the mesh",
                    outside, (long long)m);
    c.n = nn;
    h->clouds_dirty = true;
    h->need_probe = true;
    return ST_OK;
}

template <class P, class V>
int do_get_parcels(st_handle* h, int cloud, double* xyz, double* uvw, double* d)
{
    CloudBufs& c = h->clouds[cloud];
    const int64_t n = c.n;
    if (n == 0) return ST_OK;
    SortBufs<P, V> b = sort_bufs<P, V>(h, c);
    {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(unpermute_cloud<P, V>(b, c.cur, n, h->stream));
        h->launches += 1;
    }
    const int o = 1 - c.cur;
    std::vector<P> hp(n);
    std::vector<V> hv(n);
    void* ps_[3] = {c.x[o], c.y[o], c.z[o]};
    for (int a = 0; a < 3; ++a) {
        CK(cudaMemcpyAsync(hp.data(), ps_[a], n * sizeof(P), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (xyz)
            for (int64_t i = 0; i < n; ++i) xyz[a * n + i] = (double)hp[i];
    }
    void* vs_[4] = {c.u[o], c.v[o], c.w[o], c.d[o]};
    for (int a = 0; a < 4; ++a) {
        double* dst = a < 3 ? (uvw ? uvw + a * n : nullptr) : d;
        if (!dst) continue;
        CK(cudaMemcpyAsync(hv.data(), vs_[a], n * sizeof(V), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int64_t i = 0; i < n; ++i) dst[i] = (double)hv[i];
    }
    return ST_OK;
}

template <class P>
int do_get_cells(st_handle* h, int cloud, int32_t* cells)
{
    CloudBufs& c = h->clouds[cloud];
    const int64_t n = c.n;
    if (n == 0) return ST_OK;
    /* the sort key buffer is free between steps */
    if (h->tet) {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(cells_unpermute(c.id[c.cur], c.cell[c.cur], n, (int32_t*)c.keys[0], h->stream));
        h->launches += 1;
    } else {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(cells_cloud<P>((const P*)c.x[c.cur], (const P*)c.y[c.cur], (const P*)c.z[c.cur],
                          c.id[c.cur], n, mesh_k<P>(h), (int32_t*)c.keys[0], nullptr, h->stream));
        h->launches += 1;
    }
    CK(cudaMemcpyAsync(cells, c.keys[0], n * sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

template <class P, class V>
int do_get_sample(st_handle* h, int cloud, int64_t m, const int32_t* ids, double* xyz,
                  double* uvw, int32_t* cells)
{
    CloudBufs& c = h->clouds[cloud];
    const size_t b_ids = ((size_t)m * sizeof(int32_t) + 255) / 256 * 256;
    const size_t b_out = (size_t)m * 6 * sizeof(double);
    int rc;
    if ((rc = ensure_stage(h, b_ids + b_out + (size_t)m * sizeof(int32_t)))) return rc;
    char* st = static_cast<char*>(h->dstage);
    int32_t* d_ids = reinterpret_cast<int32_t*>(st);
    double* d_out = reinterpret_cast<double*>(st + b_ids);
    int32_t* d_cells = reinterpret_cast<int32_t*>(st + b_ids + b_out);
    CK(cudaMemcpyAsync(d_ids, ids, (size_t)m * sizeof(int32_t), cudaMemcpyHostToDevice,
                       h->stream));
    SortBufs<P, V> b = sort_bufs<P, V>(h, c);
    {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(sample_cloud<P, V>(b, c.cur, c.n, mesh_k<P>(h), d_ids, m, d_out, d_cells, h->stream));
        h->launches += 2;
    }
    if (xyz)
        CK(cudaMemcpyAsync(xyz, d_out, (size_t)m * 3 * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
    if (uvw)
        CK(cudaMemcpyAsync(uvw, d_out + 3 * m, (size_t)m * 3 * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream));
    if (cells)
        CK(cudaMemcpyAsync(cells, d_cells, (size_t)m * sizeof(int32_t), cudaMemcpyDeviceToHost,
                           h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int check_handle(st_handle* h)
{
    if (!h) return fail(ST_ERR_INVALID_ARGUMENT, "null handle");
    return ST_OK;
}

int check_cloud(st_handle* h, int cloud)
{
    if (cloud < 0 || cloud >= h->p.n_clouds)
        return fail(ST_ERR_INVALID_ARGUMENT, "cloud %d out of range [0, %d)", cloud,
                    h->p.n_clouds);
    return ST_OK;
}

#define DISPATCH(h, FN, ...)                                                                 \
    ((h)->p.precision == ST_PREC_FP32                                                        \
         ? FN<float, float>(__VA_ARGS__)                                                     \
         : ((h)->p.precision == ST_PREC_MIXED ? FN<double, float>(__VA_ARGS__)               \
                                              : FN<double, double>(__VA_ARGS__)))

void free_cloud(CloudBufs& c)
{
    for (int k = 0; k < 2; ++k) {
        void* arrs[] = {c.x[k], c.y[k], c.z[k], c.u[k], c.v[k], c.w[k], c.d[k],
                        c.id[k], c.keys[k], c.perm[k], c.cell[k]};
        for (void* p : arrs)
            if (p) cudaFree(p);
    }
    c = CloudBufs();
}

}  // namespace

/* ------------------------------------------------------------------------------------ */
/* graph capture and autotuning                                                         */
/* ------------------------------------------------------------------------------------ */
namespace {

/* Descriptor arrays for the current buffers [0] and for the buffers after one re-sort [1]
 * (clouds of more than one parcel swap buffers), so that a captured sequence can switch
 * between them without host copies. */
template <class P, class V>
int upload_clouds_pair(st_handle* h)
{
    int rc;
    if ((rc = upload_clouds<P, V>(h))) return rc;
    const int nc = h->p.n_clouds;
    std::vector<CloudK<P, V>> v(2 * nc);
    memcpy(v.data(), h->hclouds.data(), sizeof(CloudK<P, V>) * nc);
    for (int c = 0; c < nc; ++c) {
        CloudBufs& b = h->clouds[c];
        CloudK<P, V> k = v[c];
        if (b.n > 1) {
            const int o = 1 - b.cur;
            k.x = (P*)b.x[o]; k.y = (P*)b.y[o]; k.z = (P*)b.z[o];
            k.u = (V*)b.u[o]; k.v = (V*)b.v[o]; k.w = (V*)b.w[o]; k.d = (const V*)b.d[o];
            k.cell = b.cell[o];
        }
        v[nc + c] = k;
    }
    h->hclouds2.resize(sizeof(CloudK<P, V>) * 2 * nc);
    memcpy(h->hclouds2.data(), v.data(), h->hclouds2.size());
    if (!h->dclouds2) CK(cudaMalloc(&h->dclouds2, 2 * 256 * (size_t)nc));
    CK(cudaMemcpyAsync(h->dclouds2, v.data(), sizeof(CloudK<P, V>) * 2 * nc,
                       cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

void release_graph(st_handle* h)
{
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->gexec = nullptr;
    h->graph = nullptr;
    h->graph_steps = 0;
}

template <class P, class V>
int graph_capture(st_handle* h, int n, double dt, const double* fs)
{
    int rc;
    release_graph(h);
    /* the capture runs the finalize in stream order: nothing may still run on fin_stream */
    if ((rc = drain_fin(h))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    const bool det = (h->dep == DEP_DET1 || h->dep == DEP_DET2);
    if (det && (h->need_probe || dt != h->last_dt)) {
        /* the first-step scale comes from a read-only probe, run outside the graph */
        if ((rc = upload_clouds<P, V>(h))) return rc;
        StepArgs<P, V> a;
        a.mesh = mesh_k<P>(h);
        a.phys = phys_k<V>(h);
        a.dtP = (P)dt / (P)h->p.n_substeps;
        a.dtV = (V)a.dtP;
        split_fluid_scale<P, V>(fs ? fs[0] : 1.0, a.fscale, a.fscale_lo);
        a.nclouds = h->p.n_clouds;
        a.U = (const V*)h->dU;
        a.clouds = (const CloudK<P, V>*)h->dclouds;
        a.ctl = h->dctl;
        a.total_tiles = h->total_tiles;
        memcpy(&a.one, h->hclouds.data(), sizeof(CloudK<P, V>));
        if (a.total_tiles > 0) {
            CK(launch_step<P, V>(a, DEP_PROBE, h->grid, h->block, h->stream));
            CK(launch_set_scale(h->dctl, h->p.n_clouds, h->stream));
            h->launches += 2;
        }
        h->need_probe = false;
        h->last_dt = dt;
    }
    if ((rc = upload_clouds_pair<P, V>(h))) return rc;
    std::vector<int> cur(h->clouds.size());
    for (size_t c = 0; c < h->clouds.size(); ++c) cur[c] = h->clouds[c].cur;
    const int64_t steps0 = h->steps, launches0 = h->launches;
    const int since0 = h->steps_since_sort;
    const bool prof = h->prof;
    h->prof = false;
    CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    h->capturing = true;
    h->cap_parity = 0;
    for (int k = 0; k < n && rc == ST_OK; ++k) rc = do_step<P, V>(h, dt, fs ? fs[k] : 1.0);
    h->capturing = false;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->stream, &g);
    h->prof = prof;
    const int64_t per = h->launches - launches0;
    for (size_t c = 0; c < h->clouds.size(); ++c) h->clouds[c].cur = cur[c];
    h->steps = steps0;
    h->steps_since_sort = since0;
    h->launches = launches0;
    h->clouds_dirty = true;
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return fail(ST_ERR_CUDA, "stream capture: %s", cudaGetErrorString(e));
    h->graph = g;
    if ((e = cudaGraphInstantiate(&h->gexec, g, 0)) != cudaSuccess) {
        release_graph(h);
        return fail(ST_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(e));
    }
    h->graph_steps = n;
    h->graph_launches = per;
    return ST_OK;
}

int occupancy_grid(st_handle* h, int block)
{
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    int occ = h->p.precision == ST_PREC_FP32
                  ? step_max_active_blocks<float, float>(h->dep, block)
                  : (h->p.precision == ST_PREC_MIXED
                         ? step_max_active_blocks<double, float>(h->dep, block)
                         : step_max_active_blocks<double, double>(h->dep, block));
    return nsm * (occ < 1 ? 1 : occ);
}

}  // namespace

/* ------------------------------------------------------------------------------------ */
/* adjoint of the time-averaged source                                                  */
/* ------------------------------------------------------------------------------------ */
namespace {

int adj_check(st_handle* h, int cloud, const st_adjoint_desc* d)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (!d) return fail(ST_ERR_INVALID_ARGUMENT, "null adjoint descriptor");
    if (h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "the adjoint supports cuboid meshes only");
    if (h->p.precision == ST_PREC_FP32 || h->p.drag_model != ST_DRAG_SCHILLER_NAUMANN ||
        h->p.n_substeps != 1)
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "the adjoint supports Schiller-Naumann drag, one substep and mixed or FP64 "
                    "precision");
    if (d->n_steps < 1 || d->checkpoint_interval < 1)
        return fail(ST_ERR_INVALID_ARGUMENT, "n_steps and checkpoint_interval must be >= 1");
    if (!(d->dt > 0) || !(d->dt < 1e300)) return fail(ST_ERR_INVALID_ARGUMENT, "dt must be positive");
    if (!(h->p.drag_multiplier > 0) || !(h->p.diameter_scale > 0))
        return fail(ST_ERR_INVALID_ARGUMENT, "drag_multiplier and diameter_scale must be positive");
    return ST_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

template <class P, class V>
int adj_prepare(st_handle* h, int cloud, const st_adjoint_desc* d)
{
    AdjTape& t = h->adj;
    const int64_t n = h->clouds[cloud].n;
    const int T = d->n_steps, C = d->checkpoint_interval;
    const int nseg = (T + C - 1) / C;
    const int grid = (int)((n + 255) / 256);
    const int limbs = sizeof(V) == 8 ? 2 : 1;
    size_t off = 0;
    auto carve = [&](size_t b) { size_t o = off; off += align256(b); return o; };
    const size_t o_ckx = carve((size_t)nseg * 3 * n * sizeof(P));
    const size_t o_ckv = carve((size_t)nseg * 3 * n * sizeof(V));
    const size_t o_rv = carve((size_t)C * 3 * n * sizeof(V));
    const size_t o_rc = carve((size_t)C * n * sizeof(int32_t));
    const size_t o_rb = carve((size_t)C * n);
    const size_t o_G = carve((size_t)h->stride * sizeof(double));
    const size_t o_av = carve((size_t)3 * n * sizeof(V));
    const size_t o_pa = carve((size_t)nseg * (grid > 0 ? grid : 1) * 2 * sizeof(double));
    const size_t o_fs = carve((size_t)2 * T * sizeof(V));   /* fs, then fs_lo */
    const size_t o_mean = carve((size_t)h->stride * sizeof(double));
    const size_t o_ctl = carve(sizeof(CloudCtl));
    const size_t o_acc = carve((size_t)h->stride * limbs * 8);
    if (off > t.bytes) {
        if (t.mem) cudaFree(t.mem);
        t.mem = nullptr;
        t.bytes = 0;
        CK(cudaMalloc(&t.mem, off));
        t.bytes = off;
    }
    char* b = static_cast<char*>(t.mem);
    t.ck_x = b + o_ckx; t.ck_v = b + o_ckv; t.rec_v = b + o_rv;
    t.rec_c = reinterpret_cast<int32_t*>(b + o_rc);
    t.rec_b = reinterpret_cast<uint8_t*>(b + o_rb);
    t.G = reinterpret_cast<double*>(b + o_G);
    t.adj_v = b + o_av;
    t.partials = reinterpret_cast<double*>(b + o_pa);
    t.fsd = b + o_fs;
    t.mean = reinterpret_cast<double*>(b + o_mean);
    t.ctl = reinterpret_cast<CloudCtl*>(b + o_ctl);
    t.acc = reinterpret_cast<unsigned long long*>(b + o_acc);
    t.cloud = cloud; t.T = T; t.C = C; t.nseg = nseg; t.grid = grid; t.limbs = limbs;
    t.n = n; t.dt = d->dt;
    t.fs.assign(T, 1.0);
    if (d->fluid_scale)
        for (int k = 0; k < T; ++k) t.fs[k] = d->fluid_scale[k];
    std::vector<V> fsv(2 * (size_t)T);
    for (int k = 0; k < T; ++k) split_fluid_scale<P, V>(t.fs[k], fsv[k], fsv[T + k]);
    CK(cudaMemcpyAsync(t.fsd, fsv.data(), 2 * (size_t)T * sizeof(V), cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

template <class P, class V>
AdjArgs<P, V> adj_args(st_handle* h)
{
    AdjTape& t = h->adj;
    CloudBufs& c = h->clouds[t.cloud];
    AdjArgs<P, V> a;
    a.mesh = mesh_k<P>(h);
    a.phys = phys_k<V>(h);
    a.dtP = (P)t.dt;
    a.dtV = (V)a.dtP;
    a.n = t.n; a.T = t.T; a.C = t.C; a.limbs = t.limbs;
    a.x = (const P*)c.x[c.cur]; a.y = (const P*)c.y[c.cur]; a.z = (const P*)c.z[c.cur];
    a.u = (const V*)c.u[c.cur]; a.v = (const V*)c.v[c.cur]; a.w = (const V*)c.w[c.cur];
    a.d = (const V*)c.d[c.cur];
    a.U = (const V*)h->dU;
    a.fs = (const V*)t.fsd;
    a.fs_lo = (const V*)t.fsd + t.T;
    a.acc = t.acc; a.ctl = t.ctl;
    a.ck_x = (P*)t.ck_x; a.ck_v = (V*)t.ck_v;
    a.rec_v = (V*)t.rec_v; a.rec_c = t.rec_c; a.rec_b = t.rec_b;
    a.G = t.G; a.adj_v = (V*)t.adj_v; a.partials = t.partials;
    return a;
}

template <class P, class V>
int adj_forward(st_handle* h, int cloud, const st_adjoint_desc* d, double* mean_out)
{
    int rc;
    h->adj.valid = false;
    if ((rc = adj_prepare<P, V>(h, cloud, d))) return rc;
    AdjTape& t = h->adj;
    CloudCtl c0;
    memset(&c0, 0, sizeof c0);
    c0.emax = EXP_NONE;
    int64_t bound = t.n * (int64_t)t.T;
    if (bound < 2) bound = 2;
    c0.H = t.limbs == 1 ? 62 - QUANT_GROWTH_BITS - quant_nbits(bound) : 62 - QUANT_GROWTH_BITS;
    CK(cudaMemcpyAsync(t.ctl, &c0, sizeof c0, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(t.acc, 0, (size_t)h->stride * t.limbs * 8, h->stream));
    AdjArgs<P, V> a = adj_args<P, V>(h);
    {
        ProfScope ps(h, ST_KERNEL_ADJ_FORWARD);
        CK(launch_adj_forward<P, V>(a, true, h->stream));
        CK(launch_adj_scale(t.ctl, h->stream));
        CK(launch_adj_forward<P, V>(a, false, h->stream));
        CK(launch_adj_mean(t.acc, t.ctl, t.limbs, t.T, t.mean, h->ncells * 3, h->stream));
        h->launches += 4;
    }
    CloudCtl out;
    CK(cudaMemcpyAsync(&out, t.ctl, sizeof out, cudaMemcpyDeviceToHost, h->stream));
    if (mean_out)
        CK(cudaMemcpyAsync(mean_out, t.mean, h->ncells * 3 * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (out.lost) return fail(ST_ERR_PARCEL_OUTSIDE, "parcel(s) left the mesh in the forward pass");
    if (out.overflow)
        return fail(ST_ERR_SOURCE_RANGE, "mean-source deposit(s) exceeded the fixed-point range");
    t.valid = true;
    return ST_OK;
}

template <class P, class V>
int adj_pullback(st_handle* h, int cloud, const st_adjoint_desc* d, const double* cot,
                 double* dalpha, double* dscale, double* dv0)
{
    AdjTape& t = h->adj;
    bool same = t.valid && t.cloud == cloud && t.T == d->n_steps &&
                t.C == d->checkpoint_interval && t.dt == d->dt && t.n == h->clouds[cloud].n;
    for (int k = 0; same && k < t.T; ++k)
        same = t.fs[k] == (d->fluid_scale ? d->fluid_scale[k] : 1.0);
    if (!same)
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "st_mean_source_pullback needs a preceding st_mean_source_forward with the "
                    "same cloud and descriptor");
    const int64_t ncomp = h->ncells * 3;
    std::vector<double> G(ncomp);
    for (int64_t j = 0; j < ncomp; ++j) G[j] = cot[j] / (double)t.T;
    CK(cudaMemcpyAsync(t.G, G.data(), ncomp * sizeof(double), cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaMemsetAsync(t.adj_v, 0, (size_t)3 * t.n * sizeof(V), h->stream));
    AdjArgs<P, V> a = adj_args<P, V>(h);
    {
        ProfScope ps(h, ST_KERNEL_ADJ_REVERSE);
        for (int seg = t.nseg - 1; seg >= 0; --seg) {
            const int len = std::min(t.C, t.T - seg * t.C);
            CK(launch_adj_reverse<P, V>(a, seg, len, t.grid, h->stream));
            h->launches += 1;
        }
    }
    std::vector<double> parts((size_t)t.nseg * t.grid * 2);
    if (!parts.empty())
        CK(cudaMemcpyAsync(parts.data(), t.partials, parts.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, h->stream));
    std::vector<V> av(dv0 ? (size_t)3 * t.n : 0);
    std::vector<int32_t> id(dv0 ? t.n : 0);
    CloudBufs& c = h->clouds[cloud];
    if (dv0 && t.n > 0) {
        CK(cudaMemcpyAsync(av.data(), t.adj_v, av.size() * sizeof(V), cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaMemcpyAsync(id.data(), c.id[c.cur], id.size() * sizeof(int32_t),
                           cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    double sa = 0.0, ss = 0.0;  /* fixed order: segment, then block */
    for (size_t k = 0; k < parts.size(); k += 2) {
        sa += parts[k];
        ss += parts[k + 1];
    }
    if (dalpha) *dalpha = sa;
    if (dscale) *dscale = ss;
    if (dv0)
        for (int comp = 0; comp < 3; ++comp)
            for (int64_t j = 0; j < t.n; ++j)
                dv0[comp * t.n + id[j]] = (double)av[comp * t.n + j];
    return ST_OK;
}

}  // namespace

/* ------------------------------------------------------------------------------------ */
/* public API                                                                           */
/* ------------------------------------------------------------------------------------ */
/* Host-side staging grows with the parcel count; an allocation failure becomes a status
 * instead of an exception crossing the C ABI. */
template <class F>
static int guard_host_alloc(const char* what, F&& body)
{
    try {
        return body();
    } catch (const std::bad_alloc&) {
        return fail(ST_ERR_OUT_OF_MEMORY, "%s: out of host memory", what);
    }
}

extern "C" {

const char* st_version(void) { return "scaletrack-b200 0.1 sm_100a"; }

const char* st_last_error(void) { return g_err.c_str(); }

void st_params_default(st_params* p)
{
    if (!p) return;
    memset(p, 0, sizeof *p);
    p->mu_c = 1e-3;    /* setup.jl:12 */
    p->rho_c = 1e3;    /* setup.jl:13 */
    p->rho_d = 1.0;    /* setup.jl:14 */
    p->drag_model = ST_DRAG_STOKES_IMPLICIT;
    p->precision = ST_PREC_FP32;
    p->deposit = ST_DEPOSIT_DETERMINISTIC;
    p->n_substeps = 10;  /* A:1260 */
    p->sort_interval = 0;
    p->n_clouds = 1;
    p->block_size = 0;
    p->grid_blocks = 0;
    p->drag_multiplier = 1.0;
    p->diameter_scale = 1.0;
}

static int create_impl(const st_params* p, const st_mesh_desc* m, int64_t ncells,
                       const st_tet_mesh_desc* tm, int device, st_handle** out)
{
    if (p->precision < ST_PREC_FP32 || p->precision > ST_PREC_FP64)
        return fail(ST_ERR_INVALID_ARGUMENT, "unknown precision %d", p->precision);
    if (p->drag_model != ST_DRAG_STOKES_IMPLICIT && p->drag_model != ST_DRAG_SCHILLER_NAUMANN)
        return fail(ST_ERR_INVALID_ARGUMENT, "unknown drag model %d", p->drag_model);
    if (p->deposit != ST_DEPOSIT_DETERMINISTIC && p->deposit != ST_DEPOSIT_ATOMIC)
        return fail(ST_ERR_INVALID_ARGUMENT, "unknown deposit mode %d", p->deposit);
    if (p->n_substeps < 1) return fail(ST_ERR_INVALID_ARGUMENT, "n_substeps must be >= 1");
    if (p->n_clouds < 1 || p->n_clouds > 4096)
        return fail(ST_ERR_INVALID_ARGUMENT, "n_clouds must be in [1, 4096]");
    if (p->sort_interval < 0) return fail(ST_ERR_INVALID_ARGUMENT, "sort_interval must be >= 0");
    if (!(p->mu_c > 0) || !(p->rho_c > 0) || !(p->rho_d > 0))
        return fail(ST_ERR_INVALID_ARGUMENT, "mu_c, rho_c and rho_d must be positive");
    if (p->block_size != 0 && (p->block_size % 32 || p->block_size < 32 || p->block_size > 256))
        return fail(ST_ERR_INVALID_ARGUMENT, "block_size must be a multiple of 32 in [32, 256]");

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(ST_ERR_CUDA, "no CUDA device available (the library has no CPU path)");
    if (device < 0 || device >= ndev)
        return fail(ST_ERR_INVALID_ARGUMENT, "device %d out of range [0, %d)", device, ndev);
    if (tm && p->precision == ST_PREC_FP32)
        return fail(ST_ERR_INVALID_ARGUMENT, "tet meshes need mixed or FP64 precision");
    DeviceGuard g(device);

    st_handle* h = new st_handle();
    h->p = *p;
    h->m = *m;
    h->tet = tm != nullptr;
    h->device = device;
    h->ncells = ncells;
    h->stride = (ncells * 3 + COMP_ALIGN - 1) / COMP_ALIGN * COMP_ALIGN;
    h->psz = p->precision == ST_PREC_FP32 ? 4 : 8;
    h->vsz = p->precision == ST_PREC_FP64 ? 8 : 4;
    if (p->deposit == ST_DEPOSIT_ATOMIC) {
        h->dep = DEP_ATOMIC;
        h->limbs = 1;
    } else if (p->precision == ST_PREC_FP64) {
        h->dep = DEP_DET2;
        h->limbs = 2;
    } else {
        h->dep = DEP_DET1;
        h->limbs = 1;
    }
    h->morton = !h->tet && m->n[0] <= 1024 && m->n[1] <= 1024 && m->n[2] <= 1024;
    if (h->morton) {
        int b = 1;
        int nmax = std::max(m->n[0], std::max(m->n[1], m->n[2]));
        while ((1 << b) < nmax) ++b;
        h->key_shift = std::max(0, b - COUNT_SORT_MAX_BITS / 3);
        h->key_bits = 3 * (b - h->key_shift);
    } else {
        const int b = quant_nbits(ncells);
        h->key_shift = std::max(0, b - COUNT_SORT_MAX_BITS);
        h->key_bits = b - h->key_shift;
    }
    h->block = p->block_size ? p->block_size : 256;
    h->clouds.resize(p->n_clouds);

    auto bail = [&](int code) {
        st_destroy(h);
        return code;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(fail(ST_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e)));
    h->own_stream = true;
    const size_t ncomp = (size_t)ncells * 3;
    const size_t cells_total = (size_t)h->stride * p->n_clouds;
    if ((e = cudaMalloc(&h->dU, ncomp * h->vsz)) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->dsrc, cells_total * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->dacc, cells_total * h->limbs * 8)) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->dctl, sizeof(CloudCtl) * p->n_clouds)) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->dcounter, sizeof(unsigned int))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->dcount, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMalloc((void**)&h->dexp, sizeof(int32_t) * p->n_clouds)) != cudaSuccess ||
        (e = cudaMalloc(&h->dclouds, 256 * (size_t)p->n_clouds)) != cudaSuccess)
        return bail(fail(e == cudaErrorMemoryAllocation ? ST_ERR_OUT_OF_MEMORY : ST_ERR_CUDA,
                         "device allocation: %s", cudaGetErrorString(e)));
    if ((e = cudaMemsetAsync(h->dU, 0, ncomp * h->vsz, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->dsrc, 0, cells_total * sizeof(double), h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->dacc, 0, cells_total * h->limbs * 8, h->stream)) != cudaSuccess ||
        (e = cudaMemsetAsync(h->dcounter, 0, sizeof(unsigned int), h->stream)) != cudaSuccess)
        return bail(fail(ST_ERR_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e)));
    {
        const size_t nb = (size_t)1 << h->key_bits;
        h->scan_bytes = count_sort_scan_bytes(h->key_bits);
        if ((e = cudaMalloc((void**)&h->dbins, nb * sizeof(uint32_t))) != cudaSuccess ||
            (e = cudaMalloc((void**)&h->doffs, nb * sizeof(uint32_t))) != cudaSuccess ||
            (e = cudaMalloc(&h->dscan, h->scan_bytes > 0 ? h->scan_bytes : 16)) != cudaSuccess)
            return bail(fail(e == cudaErrorMemoryAllocation ? ST_ERR_OUT_OF_MEMORY : ST_ERR_CUDA,
                             "device allocation: %s", cudaGetErrorString(e)));
    }
    {
        std::vector<CloudCtl> ctl(p->n_clouds);
        /* bound on the deposits one cloud makes per step: one per parcel and substep */
        for (auto& c : ctl) {
            c.L = 0;
            c.emax = EXP_NONE;
            c.H = 0;
            c.fault = 0;
            c.lost = 0;
            c.overflow = 0;
        }
        if ((e = cudaMemcpyAsync(h->dctl, ctl.data(), sizeof(CloudCtl) * p->n_clouds,
                                 cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
            return bail(fail(ST_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e)));
    }
    if (h->tet) {
        const size_t nv = (size_t)tm->n_vertices, nt = (size_t)tm->n_tets;
        if ((e = cudaMalloc((void**)&h->d_verts, nv * 3 * sizeof(double))) != cudaSuccess ||
            (e = cudaMalloc((void**)&h->d_tets, nt * 4 * sizeof(int32_t))) != cudaSuccess ||
            (e = cudaMalloc((void**)&h->d_planes, nt * 4 * sizeof(double4))) != cudaSuccess ||
            (e = cudaMalloc((void**)&h->d_planes32, nt * 4 * sizeof(float4))) != cudaSuccess ||
            (e = cudaMalloc((void**)&h->d_nbr, nt * 4 * sizeof(int32_t))) != cudaSuccess ||
            (e = cudaMalloc((void**)&h->d_hops, 8 * sizeof(unsigned long long))) != cudaSuccess)
            return bail(fail(e == cudaErrorMemoryAllocation ? ST_ERR_OUT_OF_MEMORY : ST_ERR_CUDA,
                             "device allocation: %s", cudaGetErrorString(e)));
        if ((e = cudaMemcpyAsync(h->d_verts, tm->vertices, nv * 3 * sizeof(double),
                                 cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h->d_tets, tm->tets, nt * 4 * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(h->d_nbr, tm->neighbors, nt * 4 * sizeof(int32_t),
                                 cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(h->d_hops, 0, 8 * sizeof(unsigned long long), h->stream)) !=
                cudaSuccess ||
            (e = launch_tet_planes(h->d_verts, h->d_tets, (int64_t)nt, h->d_planes,
                                   h->d_planes32, h->stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
            return bail(fail(ST_ERR_CUDA, "tet mesh set-up: %s", cudaGetErrorString(e)));
        h->launches += 1;
        /* the walk needs only the planes and the neighbours */
        cudaFree(h->d_verts);
        cudaFree(h->d_tets);
        h->d_verts = nullptr;
        h->d_tets = nullptr;
        TetMeshK& k = h->tmesh;
        k.planes = h->d_planes;
        k.planes32 = h->d_planes32;
        k.nbr = h->d_nbr;
        k.nt = (int64_t)nt;
        double xm = 0.0;
        for (int a = 0; a < 3; ++a) {
            k.origin[a] = tm->origin[a];
            k.ending[a] = tm->ending[a];
            xm = std::max(xm, std::max(std::fabs(tm->origin[a]), std::fabs(tm->ending[a])));
        }
        /* rounded up to FP32: the pre-check's bound needs |x_i| <= xmax */
        float xf = (float)xm;
        if ((double)xf < xm) xf = std::nextafter(xf, INFINITY);
        k.xmax = xf;
        k.pad0 = 0;
        k.hop_limit = tm->hop_limit > 0 ? tm->hop_limit : 64;
        k.pad = 0;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    h->nsm = nsm > 0 ? nsm : 148;
    int occ = h->tet ? (p->precision == ST_PREC_FP64
                            ? step_tet_max_active_blocks<double>(h->dep, h->block)
                            : step_tet_max_active_blocks<float>(h->dep, h->block))
                     : DISPATCH(h, step_max_active_blocks, h->dep, h->block);
    if (occ < 1) occ = 1;
    h->grid = p->grid_blocks > 0 ? p->grid_blocks : nsm * occ;
    if (!h->tet && (e = DISPATCH(h, ring_prepare)) != cudaSuccess)
        return bail(fail(ST_ERR_CUDA, "ring kernel set-up: %s", cudaGetErrorString(e)));
    if (h->tet && (e = (p->precision == ST_PREC_FP64 ? tet_ring_prepare<double>()
                                                       : tet_ring_prepare<float>())) != cudaSuccess)
        return bail(fail(ST_ERR_CUDA, "ring kernel set-up: %s", cudaGetErrorString(e)));
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess)
        return bail(fail(ST_ERR_CUDA, "set-up: %s", cudaGetErrorString(e)));
    *out = h;
    return ST_OK;
}

int st_create(const st_params* p, const st_mesh_desc* m, int device, st_handle** out)
{
    if (!p || !m || !out) return fail(ST_ERR_INVALID_ARGUMENT, "null argument to st_create");
    *out = nullptr;
    for (int a = 0; a < 3; ++a) {
        if (m->n[a] < 1) return fail(ST_ERR_INVALID_ARGUMENT, "mesh n[%d] = %d < 1", a, m->n[a]);
        if (!(m->ending[a] > m->origin[a]))
            return fail(ST_ERR_INVALID_ARGUMENT, "mesh ending[%d] must exceed origin[%d]", a, a);
    }
    const int64_t ncells = (int64_t)m->n[0] * m->n[1] * m->n[2];
    if (ncells > INT32_MAX)
        return fail(ST_ERR_INVALID_ARGUMENT, "mesh has %lld cells; at most 2^31-1 supported",
                    (long long)ncells);
    return guard_host_alloc("st_create",
                            [&] { return create_impl(p, m, ncells, nullptr, device, out); });
}

static int create_tet_impl(const st_params* p, const st_tet_mesh_desc* tm, int device,
                           st_handle** out);

int st_create_tet(const st_params* p, const st_tet_mesh_desc* tm, int device, st_handle** out)
{
    return guard_host_alloc("st_create_tet", [&] { return create_tet_impl(p, tm, device, out); });
}

static int create_tet_impl(const st_params* p, const st_tet_mesh_desc* tm, int device,
                           st_handle** out)
{
    if (!p || !tm || !out) return fail(ST_ERR_INVALID_ARGUMENT, "null argument to st_create_tet");
    *out = nullptr;
    if (tm->n_vertices < 4 || tm->n_tets < 1 || tm->n_tets > INT32_MAX / 4 ||
        tm->n_vertices > INT32_MAX)
        return fail(ST_ERR_INVALID_ARGUMENT, "tet mesh sizes out of range (%lld vertices, %lld tets)",
                    (long long)tm->n_vertices, (long long)tm->n_tets);
    if (!tm->vertices || !tm->tets || !tm->neighbors)
        return fail(ST_ERR_INVALID_ARGUMENT, "null tet mesh array");
    if (tm->hop_limit < 0) return fail(ST_ERR_INVALID_ARGUMENT, "hop_limit must be >= 0");
    st_mesh_desc m;
    memset(&m, 0, sizeof m);
    for (int a = 0; a < 3; ++a) {
        if (!(tm->ending[a] > tm->origin[a]))
            return fail(ST_ERR_INVALID_ARGUMENT, "mesh ending[%d] must exceed origin[%d]", a, a);
        m.origin[a] = tm->origin[a];
        m.ending[a] = tm->ending[a];
        m.n[a] = 1;
    }
    /* every index the kernels follow must stay inside the arrays */
    const int64_t nt = tm->n_tets, nv = tm->n_vertices;
    for (int64_t i = 0; i < 4 * nt; ++i) {
        if (tm->tets[i] < 0 || tm->tets[i] >= nv)
            return fail(ST_ERR_INVALID_ARGUMENT, "tet %lld has vertex id %d out of range",
                        (long long)(i / 4), tm->tets[i]);
        if (tm->neighbors[i] < -1 || tm->neighbors[i] >= nt)
            return fail(ST_ERR_INVALID_ARGUMENT, "tet %lld has neighbour %d out of range",
                        (long long)(i / 4), tm->neighbors[i]);
    }
    /* canonical order: vertex ids increasing within each tet, neighbours permuted with them,
     * so both tets of a shared face build its plane from the same vertices in the same order */
    std::vector<int32_t> ct((size_t)nt * 4), cn((size_t)nt * 4);
    for (int64_t t = 0; t < nt; ++t) {
        int idx[4] = {0, 1, 2, 3};
        const int32_t* v = tm->tets + 4 * t;
        std::sort(idx, idx + 4, [v](int a, int b) { return v[a] < v[b]; });
        for (int k = 0; k < 4; ++k) {
            ct[4 * t + k] = v[idx[k]];
            cn[4 * t + k] = tm->neighbors[4 * t + idx[k]];
        }
        if (ct[4 * t] == ct[4 * t + 1] || ct[4 * t + 1] == ct[4 * t + 2] ||
            ct[4 * t + 2] == ct[4 * t + 3])
            return fail(ST_ERR_INVALID_ARGUMENT, "tet %lld repeats a vertex", (long long)t);
    }
    st_tet_mesh_desc c = *tm;
    c.tets = ct.data();
    c.neighbors = cn.data();
    return create_impl(p, &m, nt, &c, device, out);
}

int st_destroy(st_handle* h)
{
    if (!h) return ST_OK;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->fin_stream) {
        cudaStreamSynchronize(h->fin_stream);
        cudaStreamDestroy(h->fin_stream);
    }
    for (int p = 0; p < 2; ++p) {
        if (h->ev_step[p]) cudaEventDestroy(h->ev_step[p]);
        if (h->ev_fin[p]) cudaEventDestroy(h->ev_fin[p]);
    }
    for (auto& c : h->clouds) free_cloud(c);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    void* arrs[] = {h->dU, h->dsrc, h->dacc, h->dctl, h->dcounter, h->dcount, h->dclouds,
                    h->dstage, h->adj.mem, h->dclouds2, h->d_verts, h->d_tets, h->d_planes, h->d_planes32, h->d_nbr,
                    h->d_hops, h->dbins, h->doffs, h->dscan, h->dexp, h->dacc2, h->dLfin};
    for (void* p : arrs)
        if (p) cudaFree(p);
    for (auto& r : h->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : h->pool) cudaEventDestroy(e);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return ST_OK;
}

int64_t st_num_parcels(st_handle* h, int cloud)
{
    if (!h || cloud < 0 || cloud >= h->p.n_clouds) return -1;
    return h->clouds[cloud].n;
}

int64_t st_num_cells(st_handle* h) { return h ? h->ncells : -1; }

/* Headroom of the fixed-point deposit: H + G bits for the largest deposit of the previous
 * step, so that the sum of all deposits of one step fits in 63 bits. */
static int update_headroom(st_handle* h)
{
    std::vector<CloudCtl> ctl(h->p.n_clouds);
    CK(cudaMemcpyAsync(ctl.data(), h->dctl, sizeof(CloudCtl) * ctl.size(), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < h->p.n_clouds; ++c) {
        /* a sharded cloud sums the deposits of every rank: its headroom covers all of them */
        const int64_t np = std::max(h->clouds[c].n, h->clouds[c].shard_total);
        int64_t bound = np * (int64_t)h->p.n_substeps;
        if (bound < 2) bound = 2;
        ctl[c].H = h->limbs == 1 ? 62 - QUANT_GROWTH_BITS - quant_nbits(bound)
                                 : 62 - QUANT_GROWTH_BITS;
    }
    CK(cudaMemcpyAsync(h->dctl, ctl.data(), sizeof(CloudCtl) * ctl.size(), cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

static int set_parcels_impl(st_handle* h, int cloud, int64_t n, const double* xyz,
                            const double* uvw, const double* d, const int32_t* hint);

int st_set_parcels(st_handle* h, int cloud, int64_t n, const double* xyz, const double* uvw,
                   const double* d)
{
    return guard_host_alloc("st_set_parcels",
                            [&] { return set_parcels_impl(h, cloud, n, xyz, uvw, d, nullptr); });
}

int st_append_parcels(st_handle* h, int cloud, int64_t m, const double* xyz, const double* uvw,
                      const double* d)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "st_append_parcels fills cuboid meshes");
    if (m < 0 || h->clouds[cloud].n + m > INT32_MAX)
        return fail(ST_ERR_INVALID_ARGUMENT, "parcel count out of range");
    if (m == 0) return ST_OK;
    if (!xyz || !uvw || !d) return fail(ST_ERR_INVALID_ARGUMENT, "null parcel array");
    DeviceGuard g(h->device);
    CK(cudaStreamSynchronize(h->stream));
    release_graph(h);
    rc = guard_host_alloc("st_append_parcels",
                          [&] { return DISPATCH(h, do_append_parcels, h, cloud, m, xyz, uvw,
                                                d); });
    if (rc) return rc;
    return update_headroom(h);
}

int st_init_parcels(st_handle* h, int cloud, int64_t n, uint64_t seed, double d_min,
                    double d_max)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "st_init_parcels fills cuboid meshes");
    if (n < 0 || n > INT32_MAX)
        return fail(ST_ERR_INVALID_ARGUMENT, "parcel count %lld out of range", (long long)n);
    if (!(d_min > 0) || !(d_max >= d_min) || !(d_max < 1e300))
        return fail(ST_ERR_INVALID_ARGUMENT, "diameters must satisfy 0 < d_min <= d_max");
    DeviceGuard g(h->device);
    CK(cudaStreamSynchronize(h->stream));
    release_graph(h);
    const InitSpec spec = {seed, d_min, d_max};
    rc = DISPATCH(h, do_set_parcels, h, cloud, n, nullptr, nullptr, nullptr, nullptr, &spec);
    if (rc) return rc;
    return update_headroom(h);
}

int st_set_parcels_tet(st_handle* h, int cloud, int64_t n, const double* xyz, const double* uvw,
                       const double* d, const int32_t* hint)
{
    if (h && !h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "st_set_parcels_tet on a cuboid mesh");
    return guard_host_alloc("st_set_parcels_tet",
                            [&] { return set_parcels_impl(h, cloud, n, xyz, uvw, d, hint); });
}

int st_tet_hop_histogram(st_handle* h, uint64_t out[8], int reset)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "st_tet_hop_histogram on a cuboid mesh");
    DeviceGuard g(h->device);
    unsigned long long v[8];
    CK(cudaMemcpyAsync(v, h->d_hops, sizeof v, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (out)
        for (int k = 0; k < 8; ++k) out[k] = v[k];
    if (reset) CK(cudaMemsetAsync(h->d_hops, 0, sizeof v, h->stream));
    return ST_OK;
}

static int set_parcels_impl(st_handle* h, int cloud, int64_t n, const double* xyz,
                            const double* uvw, const double* d, const int32_t* hint)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (n < 0 || n > INT32_MAX)
        return fail(ST_ERR_INVALID_ARGUMENT, "parcel count %lld out of range", (long long)n);
    if (n > 0 && (!xyz || !uvw || !d))
        return fail(ST_ERR_INVALID_ARGUMENT, "null parcel array");
    DeviceGuard g(h->device);
    CK(cudaStreamSynchronize(h->stream));
    release_graph(h);
    std::vector<int32_t> zeros;
    if (h->tet && !hint && n > 0) {
        zeros.assign((size_t)n, 0);
        hint = zeros.data();
    }
    rc = DISPATCH(h, do_set_parcels, h, cloud, n, xyz, uvw, d, hint);
    if (rc) return rc;
    return update_headroom(h);
}

int st_get_parcels(st_handle* h, int cloud, double* xyz, double* uvw, double* d)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    DeviceGuard g(h->device);
    if ((rc = check_device_errors(h))) {
        /* still hand back the state: lost parcels were left unchanged */
        int rc2 = guard_host_alloc(
            "st_get_parcels", [&] { return DISPATCH(h, do_get_parcels, h, cloud, xyz, uvw, d); });
        return rc2 ? rc2 : rc;
    }
    return guard_host_alloc("st_get_parcels",
                            [&] { return DISPATCH(h, do_get_parcels, h, cloud, xyz, uvw, d); });
}

int st_get_cells(st_handle* h, int cloud, int32_t* cells)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (!cells && h->clouds[cloud].n > 0) return fail(ST_ERR_INVALID_ARGUMENT, "null cells");
    DeviceGuard g(h->device);
    int err = check_device_errors(h);
    rc = guard_host_alloc("st_get_cells", [&] {
        return h->p.precision == ST_PREC_FP32 ? do_get_cells<float>(h, cloud, cells)
                                              : do_get_cells<double>(h, cloud, cells);
    });
    return rc ? rc : err;
}

int st_get_parcel_sample(st_handle* h, int cloud, int64_t m, const int32_t* ids, double* xyz,
                         double* uvw, int32_t* cells)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    const int64_t n = h->clouds[cloud].n;
    if (m < 0 || (m > 0 && !ids))
        return fail(ST_ERR_INVALID_ARGUMENT, "st_get_parcel_sample: bad sample size or ids");
    for (int64_t j = 0; j < m; ++j)
        if (ids[j] < 0 || ids[j] >= n)
            return fail(ST_ERR_INVALID_ARGUMENT,
                        "st_get_parcel_sample: ids[%lld] = %d is not a parcel index (n = %lld)",
                        (long long)j, ids[j], (long long)n);
    if (m == 0) return ST_OK;
    DeviceGuard g(h->device);
    return guard_host_alloc("st_get_parcel_sample", [&] {
        return DISPATCH(h, do_get_sample, h, cloud, m, ids, xyz, uvw, cells);
    });
}

int st_get_order(st_handle* h, int cloud, int32_t* ids)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    const CloudBufs& c = h->clouds[cloud];
    if (c.n == 0) return ST_OK;
    if (!ids) return fail(ST_ERR_INVALID_ARGUMENT, "null ids");
    DeviceGuard g(h->device);
    CK(cudaMemcpyAsync(ids, c.id[c.cur], c.n * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

static int set_fluid(st_handle* h, const void* U, int elem_bytes, bool device)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!U) return fail(ST_ERR_INVALID_ARGUMENT, "null U");
    if (elem_bytes != 4 && elem_bytes != 8)
        return fail(ST_ERR_INVALID_ARGUMENT, "elem_bytes must be 4 or 8, got %d", elem_bytes);
    DeviceGuard g(h->device);
    const int64_t ncomp = h->ncells * 3;
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if ((size_t)elem_bytes == h->vsz) {
        CK(cudaMemcpyAsync(h->dU, U, ncomp * elem_bytes, kind, h->stream));
    } else {
        if ((rc = ensure_stage(h, ncomp * elem_bytes))) return rc;
        CK(cudaMemcpyAsync(h->dstage, U, ncomp * elem_bytes, kind, h->stream));
        ProfScope ps(h, ST_KERNEL_OTHER);
        if (elem_bytes == 8) CK(launch_f64_to_f32((const double*)h->dstage, (float*)h->dU, ncomp, h->stream));
        else CK(launch_f32_to_f64((const float*)h->dstage, (double*)h->dU, ncomp, h->stream));
        h->launches += 1;
    }
    if (!device) CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_set_fluid_velocity(st_handle* h, const void* U, int elem_bytes)
{
    return set_fluid(h, U, elem_bytes, false);
}

int st_set_fluid_velocity_device(st_handle* h, const void* U, int elem_bytes)
{
    return set_fluid(h, U, elem_bytes, true);
}

int st_step(st_handle* h, double dt, double fluid_scale)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!(dt > 0) || !(dt < 1e300))
        return fail(ST_ERR_INVALID_ARGUMENT, "dt must be positive and finite, got %g", dt);
    if (!(fluid_scale == fluid_scale) || fluid_scale > 1e300 || fluid_scale < -1e300)
        return fail(ST_ERR_INVALID_ARGUMENT, "fluid_scale must be finite");
    DeviceGuard g(h->device);
    return DISPATCH(h, do_step, h, dt, fluid_scale);
}

static int copy_source(st_handle* h, int cloud, void* S, int elem_bytes, bool sync)
{
    const int64_t ncomp = h->ncells * 3;
    const double* src = h->dsrc + (int64_t)cloud * h->stride;
    int rc;
    if ((rc = join_fin(h))) return rc;
    if (elem_bytes == 8) {
        CK(cudaMemcpyAsync(S, src, ncomp * 8, cudaMemcpyDeviceToHost, h->stream));
    } else {
        if ((rc = ensure_stage(h, ncomp * 4))) return rc;
        {
            ProfScope ps(h, ST_KERNEL_OTHER);
            CK(launch_f64_to_f32(src, (float*)h->dstage, ncomp, h->stream));
            h->launches += 1;
        }
        CK(cudaMemcpyAsync(S, h->dstage, ncomp * 4, cudaMemcpyDeviceToHost, h->stream));
    }
    if (sync) CK(cudaStreamSynchronize(h->stream));
    return ST_OK;
}

int st_get_source(st_handle* h, int cloud, void* S, int elem_bytes)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (!S) return fail(ST_ERR_INVALID_ARGUMENT, "null S");
    if (elem_bytes != 4 && elem_bytes != 8)
        return fail(ST_ERR_INVALID_ARGUMENT, "elem_bytes must be 4 or 8, got %d", elem_bytes);
    DeviceGuard g(h->device);
    if ((rc = copy_source(h, cloud, S, elem_bytes, true))) return rc;
    return check_device_errors(h);
}

const double* st_source_device(st_handle* h, int cloud)
{
    if (!h || cloud < 0 || cloud >= h->p.n_clouds) return nullptr;
    DeviceGuard g(h->device);
    if (join_fin(h)) return nullptr;   /* the handle's stream now follows the last source */
    return h->dsrc + (int64_t)cloud * h->stride;
}

int st_synchronize(st_handle* h)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    DeviceGuard g(h->device);
    if ((rc = join_fin(h))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    return check_device_errors(h);
}

void* st_get_stream(st_handle* h) { return h ? (void*)h->stream : nullptr; }

int st_set_stream(st_handle* h, void* stream)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    DeviceGuard g(h->device);
    if ((rc = drain_fin(h))) return rc;
    CK(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return ST_OK;
}

int st_profile_enable(st_handle* h, int on)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    h->prof = on != 0;
    return ST_OK;
}

int st_profile_read(st_handle* h, int kind, int64_t* launches, double* ms, int reset)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (kind < 0 || kind >= ST_KERNEL_KINDS)
        return fail(ST_ERR_INVALID_ARGUMENT, "unknown kernel kind %d", kind);
    DeviceGuard g(h->device);
    if ((rc = drain_fin(h))) return rc;   /* finalize events are recorded on fin_stream */
    CK(cudaStreamSynchronize(h->stream));
    cudaError_t err = cudaSuccess;
    for (auto& r : h->recs) {
        float t = 0.f;
        const cudaError_t e = cudaEventElapsedTime(&t, r.a, r.b);
        if (e == cudaSuccess) {
            h->prof_ms[r.kind] += t;
            h->prof_launches[r.kind] += 1;
        } else if (err == cudaSuccess) {
            err = e;
        }
        h->pool.push_back(r.a);
        h->pool.push_back(r.b);
    }
    h->recs.clear();
    if (err != cudaSuccess)
        return fail(ST_ERR_CUDA, "cudaEventElapsedTime: %s", cudaGetErrorString(err));
    if (launches) *launches = h->prof_launches[kind];
    if (ms) *ms = h->prof_ms[kind];
    if (reset) {
        for (int k = 0; k < ST_KERNEL_KINDS; ++k) {
            h->prof_ms[k] = 0;
            h->prof_launches[k] = 0;
        }
    }
    return ST_OK;
}

int64_t st_launch_count(st_handle* h) { return h ? h->launches : -1; }

int st_set_drag_parameters(st_handle* h, double drag_multiplier, double diameter_scale)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!(drag_multiplier > 0.0 && drag_multiplier < INFINITY) ||
        !(diameter_scale > 0.0 && diameter_scale < INFINITY))
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "st_set_drag_parameters: drag_multiplier and diameter_scale must be finite "
                    "and > 0 (got %g, %g)", drag_multiplier, diameter_scale);
    h->p.drag_multiplier = drag_multiplier;
    h->p.diameter_scale = diameter_scale;
    h->need_probe = true;      /* the deposits change size: new first-step scale */
    h->adj.valid = false;      /* the pull-back needs the forward of these parameters */
    return ST_OK;
}

int st_shard_set_total(st_handle* h, int cloud, int64_t n_parcels_all_ranks)
{
    int rc;
    if ((rc = check_handle(h)) || (rc = check_cloud(h, cloud))) return rc;
    if (n_parcels_all_ranks < 0 || n_parcels_all_ranks > ((int64_t)1 << 40))
        return fail(ST_ERR_INVALID_ARGUMENT, "st_shard_set_total: count out of range");
    if (h->dep != DEP_DET1 && h->dep != DEP_DET2)
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "sharded steps need the deterministic deposit (integer accumulators)");
    h->clouds[cloud].shard_total = n_parcels_all_ranks;
    DeviceGuard g(h->device);
    if ((rc = update_headroom(h))) return rc;
    h->need_probe = true;
    return ST_OK;
}

int st_shard_buffers(st_handle* h, void** accumulators, int64_t* n_accumulators,
                     int32_t** exponents, int32_t* n_exponents)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (accumulators) *accumulators = h->dacc;
    if (n_accumulators) *n_accumulators = h->stride * h->p.n_clouds * h->limbs;
    if (exponents) *exponents = h->dexp;
    if (n_exponents) *n_exponents = h->p.n_clouds;
    return ST_OK;
}

int st_shard_needs_probe(st_handle* h, double dt)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    return (h->need_probe || dt != h->last_dt) ? 1 : 0;
}

static int shard_phase(st_handle* h, double dt, double fs, int phase)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (h->capturing) return fail(ST_ERR_INVALID_ARGUMENT, "sharded steps cannot be captured");
    if (phase != PH_FINISH && !(dt > 0.0 && dt < INFINITY))
        return fail(ST_ERR_INVALID_ARGUMENT, "dt must be finite and > 0");
    DeviceGuard g(h->device);
    return DISPATCH(h, do_step, h, dt, fs, phase);
}

int st_shard_probe(st_handle* h, double dt, double fluid_scale)
{
    return shard_phase(h, dt, fluid_scale, PH_PROBE);
}

int st_shard_deposit(st_handle* h, double dt, double fluid_scale)
{
    return shard_phase(h, dt, fluid_scale, PH_DEPOSIT);
}

int st_shard_finish(st_handle* h)
{
    return shard_phase(h, h ? h->last_dt : 0.0, 1.0, PH_FINISH);
}

int st_set_finalize_overlap(st_handle* h, int on)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    DeviceGuard g(h->device);
    if ((rc = drain_fin(h))) return rc;
    h->fin_overlap = on != 0;
    return ST_OK;
}

int st_set_wait_limit(st_handle* h, int64_t cycles, int stall)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (cycles < 0) return fail(ST_ERR_INVALID_ARGUMENT, "st_set_wait_limit: cycles < 0");
    if (stall && cycles == 0)
        return fail(ST_ERR_INVALID_ARGUMENT, "st_set_wait_limit: a stall test needs cycles > 0");
    h->wait_cycles = stall ? -cycles : cycles;
    return ST_OK;
}

int st_set_step_kernel(st_handle* h, int kind)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (kind != ST_STEP_KERNEL_RING && kind != ST_STEP_KERNEL_WARP)
        return fail(ST_ERR_INVALID_ARGUMENT, "st_set_step_kernel: unknown kind %d", kind);
    h->ring = (kind == ST_STEP_KERNEL_RING);
    return ST_OK;
}

int st_mean_source_forward(st_handle* h, int cloud, const st_adjoint_desc* desc,
                           double* mean_source)
{
    int rc;
    if ((rc = adj_check(h, cloud, desc))) return rc;
    DeviceGuard g(h->device);
    CK(cudaStreamSynchronize(h->stream));
    return guard_host_alloc("st_mean_source_forward", [&] {
        return h->p.precision == ST_PREC_MIXED
                   ? adj_forward<double, float>(h, cloud, desc, mean_source)
                   : adj_forward<double, double>(h, cloud, desc, mean_source);
    });
}

int st_mean_source_pullback(st_handle* h, int cloud, const st_adjoint_desc* desc,
                            const double* cotangent, double* d_drag_multiplier,
                            double* d_diameter_scale, double* d_velocity0)
{
    int rc;
    if ((rc = adj_check(h, cloud, desc))) return rc;
    if (!cotangent) return fail(ST_ERR_INVALID_ARGUMENT, "null cotangent");
    DeviceGuard g(h->device);
    CK(cudaStreamSynchronize(h->stream));
    return guard_host_alloc("st_mean_source_pullback", [&] {
        return h->p.precision == ST_PREC_MIXED
                   ? adj_pullback<double, float>(h, cloud, desc, cotangent, d_drag_multiplier,
                                                 d_diameter_scale, d_velocity0)
                   : adj_pullback<double, double>(h, cloud, desc, cotangent, d_drag_multiplier,
                                                  d_diameter_scale, d_velocity0);
    });
}

int st_graph_capture(st_handle* h, int n_steps, double dt, const double* fluid_scale)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (n_steps < 1) return fail(ST_ERR_INVALID_ARGUMENT, "n_steps must be >= 1");
    if (!(dt > 0) || !(dt < 1e300)) return fail(ST_ERR_INVALID_ARGUMENT, "dt must be positive");
    if (h->p.sort_interval > 0 &&
        (h->steps_since_sort != 0 || n_steps % (2 * h->p.sort_interval) != 0))
        return fail(ST_ERR_INVALID_ARGUMENT,
                    "with re-sorting, capture right after a re-sort (or set-up) and a multiple "
                    "of 2 x sort_interval steps, so that every replay starts from the same "
                    "buffers");
    DeviceGuard g(h->device);
    return DISPATCH(h, graph_capture, h, n_steps, dt, fluid_scale);
}

int st_graph_launch(st_handle* h)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!h->gexec) return fail(ST_ERR_INVALID_ARGUMENT, "no captured graph");
    DeviceGuard g(h->device);
    /* the graph deposits into the first accumulator in stream order: pending overlapped
     * finalizes (which clear it) come first */
    if ((rc = join_fin(h))) return rc;
    CK(cudaGraphLaunch(h->gexec, h->stream));
    h->steps += h->graph_steps;
    h->launches += h->graph_launches;
    return ST_OK;
}

int st_graph_release(st_handle* h)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    DeviceGuard g(h->device);
    cudaStreamSynchronize(h->stream);
    release_graph(h);
    return ST_OK;
}

static int autotune_impl(st_handle* h, double dt, int trial_steps, st_tune_result* out);

int st_autotune(st_handle* h, double dt, int trial_steps, st_tune_result* out)
{
    return guard_host_alloc("st_autotune",
                            [&] { return autotune_impl(h, dt, trial_steps, out); });
}

static int autotune_impl(st_handle* h, double dt, int trial_steps, st_tune_result* out)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (trial_steps < 4) return fail(ST_ERR_INVALID_ARGUMENT, "trial_steps must be >= 4");
    if (h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "st_autotune supports cuboid meshes only");
    if (!(dt > 0) || !(dt < 1e300)) return fail(ST_ERR_INVALID_ARGUMENT, "dt must be positive");
    DeviceGuard g(h->device);
    CK(cudaStreamSynchronize(h->stream));
    release_graph(h);
    /* trials run on a copy of the handle so that the caller's state does not advance */
    st_handle* t = nullptr;
    if ((rc = st_create(&h->p, &h->m, h->device, &t))) return rc;
    for (int c = 0; c < h->p.n_clouds && rc == ST_OK; ++c) {
        const int64_t n = h->clouds[c].n;
        std::vector<double> xyz(3 * n), uvw(3 * n), d(n);
        if (n > 0 && (rc = st_get_parcels(h, c, xyz.data(), uvw.data(), d.data()))) break;
        rc = st_set_parcels(t, c, n, xyz.data(), uvw.data(), d.data());
    }
    if (rc == ST_OK) {
        cudaError_t e = cudaMemcpyAsync(t->dU, h->dU, h->ncells * 3 * h->vsz,
                                        cudaMemcpyDeviceToDevice, t->stream);
        if (e != cudaSuccess) rc = fail(ST_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e));
    }
    const int blocks[] = {128, 256};
    const int sorts[] = {0, 10, 20, 40};
    st_tune_result best;
    best.block_size = h->block;
    best.grid_blocks = h->grid;
    best.sort_interval = h->p.sort_interval;
    best.ms_per_step = 1e300;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (rc == ST_OK) {
        cudaError_t e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        if (e != cudaSuccess) rc = fail(ST_ERR_CUDA, "cudaEventCreate: %s", cudaGetErrorString(e));
    }
    for (int bi = 0; bi < 2 && rc == ST_OK; ++bi) {
        for (int si = 0; si < 4 && rc == ST_OK; ++si) {
            if (sorts[si] > trial_steps) continue;
            t->block = blocks[bi];
            t->grid = occupancy_grid(t, blocks[bi]);
            t->p.sort_interval = sorts[si];
            t->steps_since_sort = 0;
            if ((rc = DISPATCH(t, do_sort_all, t))) break;  /* every trial starts sorted */
            for (int k = 0; k < 2 && rc == ST_OK; ++k) rc = st_step(t, dt, 1.0);
            if (rc) break;
            cudaError_t e = cudaEventRecord(e0, t->stream);
            for (int k = 0; k < trial_steps && rc == ST_OK && e == cudaSuccess; ++k)
                rc = st_step(t, dt, 1.0);
            if (e == cudaSuccess) e = cudaEventRecord(e1, t->stream);
            if (rc) break;
            if ((rc = st_synchronize(t))) break;
            float ms = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) {
                rc = fail(ST_ERR_CUDA, "autotuner timing: %s", cudaGetErrorString(e));
                break;
            }
            const double per = ms / trial_steps;
            if (per < best.ms_per_step) {
                best.block_size = blocks[bi];
                best.grid_blocks = t->grid;
                best.sort_interval = sorts[si];
                best.ms_per_step = per;
            }
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    st_destroy(t);
    if (rc) return rc;
    h->block = best.block_size;
    h->grid = best.grid_blocks;
    h->p.block_size = best.block_size;
    h->p.grid_blocks = best.grid_blocks;
    h->p.sort_interval = best.sort_interval;
    h->steps_since_sort = 0;
    if (out) *out = best;
    return ST_OK;
}

/* ------------------------------------------------------------------------------------ */
/* restart files                                                                        */
/* ------------------------------------------------------------------------------------ */
/* Layout (little endian): "STSTATE1", int32 precision, n_clouds, tet flag, pad, int64
 * nCells, double last dt, int64 steps, int32 steps since the last re-sort, int32 "probe
 * pending"; per cloud int32 L, int32 H, int64 n, then double xyz[3][n], uvw[3][n], d[n] and,
 * for tet meshes, int32 owning tet[n].  Parcel order is that of st_set_parcels.  With the
 * fixed-point scale L carried over, a restarted run continues bit for bit. */
static const char ST_STATE_MAGIC[8] = {'S', 'T', 'S', 'T', 'A', 'T', 'E', '1'};

static int save_state_impl(st_handle* h, const char* path)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!path) return fail(ST_ERR_INVALID_ARGUMENT, "null path");
    DeviceGuard g(h->device);
    if ((rc = st_synchronize(h))) return rc;
    const int nc = h->p.n_clouds;
    std::vector<CloudCtl> ctl(nc);
    CK(cudaMemcpyAsync(ctl.data(), h->dctl, sizeof(CloudCtl) * nc, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    FILE* f = fopen(path, "wb");
    if (!f) return fail(ST_ERR_INVALID_ARGUMENT, "cannot open %s for writing", path);
    bool ok = fwrite(ST_STATE_MAGIC, 8, 1, f) == 1;
    const int32_t hdr[4] = {h->p.precision, nc, h->tet ? 1 : 0, 0};
    const int64_t nce = h->ncells;
    const int32_t sched[2] = {h->steps_since_sort, h->need_probe ? 1 : 0};
    ok = ok && fwrite(hdr, sizeof hdr, 1, f) == 1 && fwrite(&nce, 8, 1, f) == 1 &&
         fwrite(&h->last_dt, 8, 1, f) == 1 && fwrite(&h->steps, 8, 1, f) == 1 &&
         fwrite(sched, sizeof sched, 1, f) == 1;
    for (int c = 0; c < nc && ok; ++c) {
        const int64_t n = h->clouds[c].n;
        const int32_t lh[2] = {ctl[c].L, ctl[c].H};
        std::vector<double> xyz(3 * n), uvw(3 * n), d(n);
        if (n > 0 && (rc = DISPATCH(h, do_get_parcels, h, c, xyz.data(), uvw.data(), d.data()))) {
            fclose(f);
            return rc;
        }
        ok = fwrite(lh, sizeof lh, 1, f) == 1 && fwrite(&n, 8, 1, f) == 1;
        if (n > 0)
            ok = ok && fwrite(xyz.data(), 8, 3 * n, f) == (size_t)(3 * n) &&
                 fwrite(uvw.data(), 8, 3 * n, f) == (size_t)(3 * n) &&
                 fwrite(d.data(), 8, n, f) == (size_t)n;
        if (h->tet && n > 0) {
            std::vector<int32_t> cells(n);
            if ((rc = do_get_cells<double>(h, c, cells.data()))) {
                fclose(f);
                return rc;
            }
            ok = ok && fwrite(cells.data(), 4, n, f) == (size_t)n;
        }
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) return fail(ST_ERR_INVALID_ARGUMENT, "short write to %s", path);
    return ST_OK;
}

int st_save_state(st_handle* h, const char* path)
{
    return guard_host_alloc("st_save_state", [&] { return save_state_impl(h, path); });
}

/* Reads the whole file and checks it before the handle is touched, so a truncated or
 * inconsistent file leaves the handle as it was. */
static int load_state_impl(st_handle* h, const char* path)
{
    int rc;
    if (h && (rc = drain_fin(h))) return rc;
    struct Closer {
        FILE* f;
        ~Closer() { if (f) fclose(f); }
    } file{fopen(path, "rb")};
    FILE* f = file.f;
    if (!f) return fail(ST_ERR_INVALID_ARGUMENT, "cannot open %s", path);
    auto bad = [&](const char* why) { return fail(ST_ERR_INVALID_ARGUMENT, "%s: %s", path, why); };
    if (fseek(f, 0, SEEK_END) != 0) return bad("cannot seek");
    const long fsize = ftell(f);
    if (fsize < 0 || fseek(f, 0, SEEK_SET) != 0) return bad("cannot seek");
    char magic[8];
    int32_t hdr[4], sched[2];
    int64_t nce, steps;
    double last_dt;
    if (fread(magic, 8, 1, f) != 1 || memcmp(magic, ST_STATE_MAGIC, 8) != 0)
        return bad("not a scaletrack state file");
    if (fread(hdr, sizeof hdr, 1, f) != 1 || fread(&nce, 8, 1, f) != 1 ||
        fread(&last_dt, 8, 1, f) != 1 || fread(&steps, 8, 1, f) != 1 ||
        fread(sched, sizeof sched, 1, f) != 1)
        return bad("truncated header");
    if (hdr[0] != h->p.precision || hdr[1] != h->p.n_clouds || hdr[2] != (h->tet ? 1 : 0) ||
        nce != h->ncells)
        return bad("precision, cloud count, mesh kind or cell count differ from the handle's");
    if (steps < 0 || sched[0] < 0 || (sched[1] != 0 && sched[1] != 1) || !(last_dt >= 0.0) ||
        !(last_dt < 1e300))
        return bad("invalid step bookkeeping");
    const int nc = h->p.n_clouds;
    const int64_t per_parcel = 7 * 8 + (h->tet ? 4 : 0);
    struct Cloud {
        int32_t L = 0, H = 0;
        int64_t n = 0;
        std::vector<double> xyz, uvw, d;
        std::vector<int32_t> cells;
    };
    std::vector<Cloud> cl(nc);
    for (int c = 0; c < nc; ++c) {
        int32_t lh[2];
        int64_t n;
        if (fread(lh, sizeof lh, 1, f) != 1 || fread(&n, 8, 1, f) != 1)
            return bad("truncated cloud header");
        /* the deposit exponent lies in [-1074, 1024] and the headroom in [0, 62] */
        if (n < 0 || n > INT32_MAX || lh[1] < 0 || lh[1] > 62 || lh[0] < -1200 || lh[0] > 1100)
            return bad("invalid cloud header");
        const long here = ftell(f);
        if (here < 0 || (int64_t)(fsize - here) < n * per_parcel)
            return bad("truncated parcel data");
        Cloud& k = cl[c];
        k.L = lh[0];
        k.H = lh[1];
        k.n = n;
        k.xyz.resize(3 * n);
        k.uvw.resize(3 * n);
        k.d.resize(n);
        k.cells.resize(h->tet ? n : 0);
        if (n > 0 && (fread(k.xyz.data(), 8, 3 * n, f) != (size_t)(3 * n) ||
                      fread(k.uvw.data(), 8, 3 * n, f) != (size_t)(3 * n) ||
                      fread(k.d.data(), 8, n, f) != (size_t)n ||
                      (h->tet && fread(k.cells.data(), 4, n, f) != (size_t)n)))
            return bad("truncated parcel data");
    }
    for (int c = 0; c < nc; ++c) {
        Cloud& k = cl[c];
        if ((rc = set_parcels_impl(h, c, k.n, k.xyz.data(), k.uvw.data(), k.d.data(),
                                   h->tet ? k.cells.data() : nullptr)))
            return rc;
    }
    /* the scale of the next step and the step bookkeeping, as saved */
    DeviceGuard g(h->device);
    std::vector<CloudCtl> ctl(nc);
    CK(cudaMemcpyAsync(ctl.data(), h->dctl, sizeof(CloudCtl) * nc, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (int c = 0; c < nc; ++c) {
        ctl[c].L = cl[c].L;
        ctl[c].H = cl[c].H;
        ctl[c].emax = EXP_NONE;
    }
    CK(cudaMemcpyAsync(h->dctl, ctl.data(), sizeof(CloudCtl) * nc, cudaMemcpyHostToDevice,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->last_dt = last_dt;
    h->steps = steps;
    h->steps_since_sort = sched[0];
    h->need_probe = sched[1] != 0;
    return ST_OK;
}

int st_load_state(st_handle* h, const char* path)
{
    int rc;
    if ((rc = check_handle(h))) return rc;
    if (!path) return fail(ST_ERR_INVALID_ARGUMENT, "null path");
    return guard_host_alloc("st_load_state", [&] { return load_state_impl(h, path); });
}

/* ------------------------------------------------------------------------------------ */
/* reference-compatible shims                                                           */
/* ------------------------------------------------------------------------------------ */
struct Adopted {
    void* ptr = nullptr;
    void* dptr = nullptr;   /* the same pinned pages as the device addresses them */
    int size = 0;
    int ncomp = 0;
    int tbytes = 0;
};
static int g_exchange = ST_EXCHANGE_COPY;
static std::mutex g_mu;
static st_handle* g_default = nullptr;
static std::map<std::string, Adopted> g_arrays;

/* State of the asynchronous coupling (st_evolve_cloud_async) of the default handle. */
struct AsyncCoupling {
    bool ready = false;
    bool stepped = false;          /* a step has been launched: its source feeds the estimate */
    cudaStream_t copy = nullptr;   /* U in, beside the compute stream */
    cudaStream_t back = nullptr;   /* estimate out, concurrent with the upload (full duplex) */
    cudaEvent_t up = nullptr;      /* U of this call is on the device */
    cudaEvent_t est = nullptr;     /* estimate of this call is ready */
    cudaEvent_t down = nullptr;    /* estimate is in UTrans */
    cudaEvent_t taken = nullptr;   /* the step has its own copy of U (duraw is free) */
    double* dest = nullptr;        /* FP64 estimate, carried from call to call */
    float* dest32 = nullptr;       /* its FP32 copy for a 4-byte UTrans */
    void* duraw = nullptr;         /* U as the host holds it */
    CloudCtl* hctl = nullptr;      /* pinned copy of the control blocks */
};
static AsyncCoupling g_async;

static void async_release()
{
    AsyncCoupling& a = g_async;
    /* the compute stream may still read duraw; the copy stream may still write UTrans */
    if (g_default && g_default->stream) cudaStreamSynchronize(g_default->stream);
    if (a.copy) cudaStreamSynchronize(a.copy);
    if (a.back) cudaStreamSynchronize(a.back);
    if (a.taken) cudaEventDestroy(a.taken);
    if (a.up) cudaEventDestroy(a.up);
    if (a.est) cudaEventDestroy(a.est);
    if (a.down) cudaEventDestroy(a.down);
    if (a.copy) cudaStreamDestroy(a.copy);
    if (a.back) cudaStreamDestroy(a.back);
    if (a.dest) cudaFree(a.dest);
    if (a.dest32) cudaFree(a.dest32);
    if (a.duraw) cudaFree(a.duraw);
    if (a.hctl) cudaFreeHost(a.hctl);
    a = AsyncCoupling();
}

/* st_setup with another mesh keeps the exchange arrays (the caller may still hold them),
 * so a step checks that they were allocated for the default handle's cell count;
 * st_finalize releases them for a new allocation. */
static int check_exchange_sizes(const st_handle* h, const Adopted& U, const Adopted& S)
{
    for (const Adopted* a : {&U, &S})
        if ((int64_t)a->size != h->ncells || a->ncomp != 3)
            return fail(ST_ERR_INVALID_ARGUMENT,
                        "the exchange arrays hold %d cells, the mesh of st_setup has %lld: "
                        "call st_finalize and allocate them again", a->size,
                        (long long)h->ncells);
    return ST_OK;
}

int st_setup(const st_params* p, const st_mesh_desc* m)
{
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    st_handle* h = nullptr;
    int rc = st_create(p, m, dev, &h);
    if (rc) return rc;
    async_release();
    if (g_default) st_destroy(g_default);
    /* the coupling calls synchronise every step: nothing to overlap the finalize with */
    h->fin_overlap = false;
    g_default = h;
    return ST_OK;
}

st_handle* st_default_handle(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_default;
}

void* st_allocate_array(const char* name, int size, int nComponents, int typeByteSize)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_default) {
        fail(ST_ERR_NOT_INITIALISED, "st_allocate_array called before st_setup");
        return nullptr;
    }
    if (!name || (strcmp(name, "U") != 0 && strcmp(name, "UTrans") != 0)) {
        fail(ST_ERR_INVALID_ARGUMENT, "unknown field name '%s' (expected U or UTrans)",
             name ? name : "(null)");
        return nullptr;
    }
    if (typeByteSize != 4 && typeByteSize != 8) {  /* A:1444-1452 */
        fail(ST_ERR_INVALID_ARGUMENT,
             "size of the library's component type (4 or 8 bytes) is different from the "
             "extern type: %d", typeByteSize);
        return nullptr;
    }
    if ((int64_t)size != g_default->ncells) {      /* A:1454-1465 */
        fail(ST_ERR_INVALID_ARGUMENT, "size of the mesh: %lld is different from field's %s size: %d",
             (long long)g_default->ncells, name, size);
        return nullptr;
    }
    if (nComponents != 3) {
        fail(ST_ERR_INVALID_ARGUMENT, "field %s must have 3 components, got %d", name,
             nComponents);
        return nullptr;
    }
    auto it = g_arrays.find(name);
    if (it != g_arrays.end()) {
        Adopted& a = it->second;
        if (a.size == size && a.ncomp == nComponents && a.tbytes == typeByteSize) return a.ptr;
        fail(ST_ERR_INVALID_ARGUMENT, "field %s already allocated with a different layout", name);
        return nullptr;
    }
    Adopted a;
    DeviceGuard g(g_default->device);
    cudaError_t e = cudaHostAlloc(&a.ptr, (size_t)size * nComponents * typeByteSize,
                                  cudaHostAllocPortable | cudaHostAllocMapped);
    if (e != cudaSuccess) {
        fail(ST_ERR_CUDA, "cudaHostAlloc: %s", cudaGetErrorString(e));
        return nullptr;
    }
    if ((e = cudaHostGetDevicePointer(&a.dptr, a.ptr, 0)) != cudaSuccess) {
        cudaFreeHost(a.ptr);
        fail(ST_ERR_CUDA, "cudaHostGetDevicePointer: %s", cudaGetErrorString(e));
        return nullptr;
    }
    memset(a.ptr, 0, (size_t)size * nComponents * typeByteSize);
    a.size = size;
    a.ncomp = nComponents;
    a.tbytes = typeByteSize;
    g_arrays[name] = a;
    return a.ptr;
}

int st_evolve_cloud(double dt)
{
    std::lock_guard<std::mutex> lk(g_mu);
    st_handle* h = g_default;
    if (!h) return fail(ST_ERR_NOT_INITIALISED, "st_evolve_cloud called before st_setup");
    auto iu = g_arrays.find("U");
    auto is = g_arrays.find("UTrans");
    if (iu == g_arrays.end() || is == g_arrays.end())
        return fail(ST_ERR_NOT_INITIALISED, "U and UTrans must be allocated with "
                                            "st_allocate_array before st_evolve_cloud");
    if (int rc0 = check_exchange_sizes(h, iu->second, is->second)) return rc0;
    DeviceGuard g(h->device);
    const int64_t ncomp = h->ncells * 3;
    int rc;
    if (g_exchange == ST_EXCHANGE_MAPPED) {
        /* zero-copy: kernels read U from and write the source to the pinned pages */
        {
            ProfScope ps(h, ST_KERNEL_OTHER);
            CK(launch_convert(iu->second.dptr, iu->second.tbytes, h->dU, (int)h->vsz, ncomp,
                              h->stream));
            h->launches += 1;
        }
        if ((rc = DISPATCH(h, do_step, h, dt, 1.0))) return rc;
        /* the source is read on the handle's stream: after its conversion, wherever the
         * handle runs that (st_set_finalize_overlap) */
        if ((rc = join_fin(h))) return rc;
        {
            ProfScope ps(h, ST_KERNEL_OTHER);
            CK(launch_convert(h->dsrc, 8, is->second.dptr, is->second.tbytes, ncomp,
                              h->stream));
            h->launches += 1;
        }
        CK(cudaStreamSynchronize(h->stream));
        return check_device_errors(h);
    }
    /* U host -> device (A:1079-1083) */
    if ((size_t)iu->second.tbytes == h->vsz) {
        CK(cudaMemcpyAsync(h->dU, iu->second.ptr, ncomp * h->vsz, cudaMemcpyHostToDevice,
                           h->stream));
    } else {
        if ((rc = ensure_stage(h, ncomp * 8))) return rc;
        CK(cudaMemcpyAsync(h->dstage, iu->second.ptr, ncomp * iu->second.tbytes,
                           cudaMemcpyHostToDevice, h->stream));
        ProfScope ps(h, ST_KERNEL_OTHER);
        if (iu->second.tbytes == 8)
            CK(launch_f64_to_f32((const double*)h->dstage, (float*)h->dU, ncomp, h->stream));
        else
            CK(launch_f32_to_f64((const float*)h->dstage, (double*)h->dU, ncomp, h->stream));
        h->launches += 1;
    }
    if (is->second.tbytes == 4) {
        /* the finalize writes the 4-byte source next to the FP64 one: no conversion pass */
        const size_t b32 = (size_t)h->stride * h->p.n_clouds * sizeof(float);
        if ((rc = ensure_stage(h, b32 > (size_t)ncomp * 8 ? b32 : (size_t)ncomp * 8))) return rc;
        h->dsrc32 = static_cast<float*>(h->dstage);
        rc = DISPATCH(h, do_step, h, dt, 1.0);
        h->dsrc32 = nullptr;
        if (rc || (rc = join_fin(h))) return rc;
        /* source device -> host (A:1148-1152) */
        CK(cudaMemcpyAsync(is->second.ptr, h->dstage, ncomp * 4, cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        return check_device_errors(h);
    }
    if ((rc = DISPATCH(h, do_step, h, dt, 1.0))) return rc;
    /* source device -> host (A:1148-1152) */
    if ((rc = copy_source(h, 0, is->second.ptr, is->second.tbytes, true))) return rc;
    return check_device_errors(h);
}

/* One fluid step of the asynchronous coupling (the reference's default mode, A:1062-1190
 * with the ConstExtrapolator of A:300-316 and A:742-747).  Call k returns once U_k has been
 * taken and UTrans holds the estimate est_k = 2 S_{k-1} - est_{k-1} (est_0 = 0), where
 * S_{k-1} is the true source of the step launched by call k-1; step k itself runs on the
 * GPU while the caller solves the next fluid step.  U's upload and the estimate's download
 * go through two more streams, so they overlap the step still running and each other. */
int st_evolve_cloud_async(double dt)
{
    std::lock_guard<std::mutex> lk(g_mu);
    st_handle* h = g_default;
    if (!h) return fail(ST_ERR_NOT_INITIALISED, "st_evolve_cloud_async called before st_setup");
    auto iu = g_arrays.find("U");
    auto is = g_arrays.find("UTrans");
    if (iu == g_arrays.end() || is == g_arrays.end())
        return fail(ST_ERR_NOT_INITIALISED, "U and UTrans must be allocated with "
                                            "st_allocate_array before st_evolve_cloud_async");
    if (int rc0 = check_exchange_sizes(h, iu->second, is->second)) return rc0;
    if (!(dt > 0) || !(dt < 1e300))
        return fail(ST_ERR_INVALID_ARGUMENT, "dt must be positive and finite, got %g", dt);
    if (h->tet) return fail(ST_ERR_INVALID_ARGUMENT, "the shims drive cuboid meshes");
    DeviceGuard g(h->device);
    const int64_t ncomp = h->ncells * 3;
    const int nc = h->p.n_clouds;
    AsyncCoupling& A = g_async;
    int rc;
    if (!A.ready) {
        CK(cudaStreamCreateWithFlags(&A.copy, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&A.back, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&A.up, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&A.est, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&A.down, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&A.taken, cudaEventDisableTiming));
        CK(cudaMalloc((void**)&A.dest, ncomp * sizeof(double)));
        CK(cudaMalloc((void**)&A.dest32, ncomp * sizeof(float)));
        CK(cudaMalloc(&A.duraw, ncomp * 8));
        CK(cudaHostAlloc((void**)&A.hctl, sizeof(CloudCtl) * nc, cudaHostAllocPortable));
        CK(cudaMemsetAsync(A.dest, 0, ncomp * sizeof(double), h->stream));
        CK(cudaEventRecord(A.taken, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        A.ready = true;
    }
    /* duraw is free once the previous call's step has copied U out of it */
    CK(cudaStreamWaitEvent(A.copy, A.taken, 0));
    /* U_k in, on the copy stream (the step still running reads the handle's own U) */
    const int ub = iu->second.tbytes;
    CK(cudaMemcpyAsync(A.duraw, iu->second.ptr, ncomp * ub, cudaMemcpyHostToDevice, A.copy));
    CK(cudaEventRecord(A.up, A.copy));
    /* after step k-1: its bookkeeping, then est_k from its source (once its conversion,
     * wherever the handle runs that, has finished) */
    if ((rc = join_fin(h))) return rc;
    CK(cudaMemcpyAsync(A.hctl, h->dctl, sizeof(CloudCtl) * nc, cudaMemcpyDeviceToHost,
                       h->stream));
    {
        ProfScope ps(h, ST_KERNEL_OTHER);
        CK(launch_extrapolate(A.stepped ? h->dsrc : nullptr, A.dest,
                              is->second.tbytes == 4 ? A.dest32 : nullptr, ncomp, h->stream));
        h->launches += 1;
    }
    CK(cudaEventRecord(A.est, h->stream));
    CK(cudaStreamWaitEvent(A.back, A.est, 0));
    if (is->second.tbytes == 4)
        CK(cudaMemcpyAsync(is->second.ptr, A.dest32, ncomp * 4, cudaMemcpyDeviceToHost, A.back));
    else
        CK(cudaMemcpyAsync(is->second.ptr, A.dest, ncomp * 8, cudaMemcpyDeviceToHost, A.back));
    CK(cudaEventRecord(A.down, A.back));
    /* step k on U_k */
    CK(cudaStreamWaitEvent(h->stream, A.up, 0));
    if ((size_t)ub == h->vsz) {
        CK(cudaMemcpyAsync(h->dU, A.duraw, ncomp * ub, cudaMemcpyDeviceToDevice, h->stream));
    } else {
        ProfScope ps(h, ST_KERNEL_OTHER);
        if (ub == 8)
            CK(launch_f64_to_f32((const double*)A.duraw, (float*)h->dU, ncomp, h->stream));
        else
            CK(launch_f32_to_f64((const float*)A.duraw, (double*)h->dU, ncomp, h->stream));
        h->launches += 1;
    }
    CK(cudaEventRecord(A.taken, h->stream));
    if ((rc = DISPATCH(h, do_step, h, dt, 1.0))) return rc;
    A.stepped = true;
    /* return once U_k is taken and est_k is in UTrans; step k keeps running */
    CK(cudaEventSynchronize(A.up));
    CK(cudaEventSynchronize(A.down));
    unsigned long long lost = 0, ovf = 0;
    for (int c = 0; c < nc; ++c) {
        lost += A.hctl[c].lost;
        ovf += A.hctl[c].overflow;
    }
    if (lost || ovf) {
        /* reported once: the counters are cleared on the device, in stream order */
        CK(cudaStreamSynchronize(h->stream));
        return check_device_errors(h);
    }
    return ST_OK;
}

int st_set_exchange_mode(int mode)
{
    if (mode != ST_EXCHANGE_COPY && mode != ST_EXCHANGE_MAPPED)
        return fail(ST_ERR_INVALID_ARGUMENT, "unknown exchange mode %d", mode);
    std::lock_guard<std::mutex> lk(g_mu);
    g_exchange = mode;
    return ST_OK;
}

int st_finalize(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    g_exchange = ST_EXCHANGE_COPY;
    async_release();
    if (g_default) st_destroy(g_default);
    g_default = nullptr;
    for (auto& kv : g_arrays)
        if (kv.second.ptr) cudaFreeHost(kv.second.ptr);
    g_arrays.clear();
    return ST_OK;
}

}  // extern "C"
