/*
 * st_internal.h -- data layout shared by the host side (st_abi.cu) and the kernels.
 *
 * HBM layout (one handle):
 *   parcels, per cloud, structure of arrays, two copies (A and B) so that the Morton
 *   re-sort can gather out of place:  x,y,z : P[n]   u,v,w,d : V[n]   id : int32[n]
 *   cell velocity U        : V[nCells][3]            (the exchange layout, A:204)
 *   source                 : double[nClouds][stride]      stride = nCells*3 rounded up to 4
 *   fixed-point accumulator: uint64[nClouds][stride][limbs]   (deterministic deposit)
 *   control blocks         : CloudCtl[nClouds]
 * P is the position type and V the velocity/drag type of the precision mode.
 */
#ifndef ST_INTERNAL_H
#define ST_INTERNAL_H

#include <stdint.h>
#include <cuda_runtime.h>

namespace st {

constexpr int EXP_NONE = -100000;      /* "no deposit seen" for the max-exponent tracker */
#ifndef ST_WARP_TILE
#define ST_WARP_TILE 32
#endif
constexpr int WARP_TILE = ST_WARP_TILE; /* parcels per warp tile of the step kernel        */
constexpr int COMP_ALIGN = 4;          /* per-cloud cell-array strides are padded to this  */
constexpr int QUANT_GROWTH_BITS = 8;   /* deposits may grow 2^8 x between steps          */

enum DepMode { DEP_DET1 = 0, DEP_DET2 = 1, DEP_ATOMIC = 2, DEP_PROBE = 3 };

/* Mixed precision: FP64 positions with FP32 drag and velocities. */
template <class P, class V>
constexpr bool is_mixed = sizeof(P) == 8 && sizeof(V) == 4;

/* The fluid factor rounded to the velocity type; mixed precision also carries the FP64
 * remainder, which the slip velocity adds back (st_device.cuh slip). */
template <class P, class V>
inline void split_fluid_scale(double fs, V& hi, V& lo)
{
    hi = (V)fs;
    lo = is_mixed<P, V> ? (V)(fs - (double)hi) : (V)0;
}

template <class P>
struct MeshK {
    int32_t N[3];
    P origin[3];
    P rD[3];        /* 1/Δ per axis, formed in FP64 and rounded to P (A:237-240) */
    int32_t NxNy;
    int32_t pad;
    int64_t nCells;
};

template <class V>
struct PhysK {
    V mu;       /* carrier dynamic viscosity */
    V rho_d;    /* parcel density */
    V rr;       /* rho_d / rho_c */
    V nu;       /* carrier kinematic viscosity */
    V rnu;      /* 1/nu, formed in FP64 and rounded to V (Schiller-Naumann Re = |u-v| d / nu) */
    V alpha;    /* drag multiplier */
    V dscale;   /* diameter scale */
    int32_t drag;
    int32_t nsub;
};

/* Device-resident per-cloud control block. */
struct CloudCtl {
    int32_t L;                   /* fixed-point scale exponent of the current step        */
    int32_t emax;                /* max frexp exponent of this step's deposits            */
    int32_t H;                   /* headroom bits: first step maps 2^emax to 2^H          */
    int32_t fault;               /* bit 0: the ring kernel's producer, bit 1: a consumer gave
                                    up waiting on a pipeline barrier (sticky)              */
    unsigned long long lost;     /* parcels that could not be located (sticky)            */
    unsigned long long overflow; /* deposits beyond the fixed-point range (sticky)        */
};

template <class P, class V>
struct CloudK {
    P* x;
    P* y;
    P* z;
    V* u;
    V* v;
    V* w;
    const V* d;
    int64_t n;
    int64_t tile0;              /* first warp tile (WARP_TILE parcels) of this cloud */
    unsigned long long* acc;    /* [stride*limbs], stride = nCells*3 padded to COMP_ALIGN */
    double* src;                /* [stride] */
    int32_t* cell;              /* owning tet per parcel (tet meshes), else nullptr */
};

template <class P, class V>
struct StepArgs {
    MeshK<P> mesh;
    PhysK<V> phys;
    P dtP;                      /* substep for positions  */
    V dtV;                      /* substep for drag       */
    V fscale;                   /* factor on U            */
    V fscale_lo;                /* mixed precision: FP64 factor - fscale, else 0 */
    int32_t nclouds;
    const V* U;                 /* [nCells*3] */
    const CloudK<P, V>* clouds; /* [nclouds] device array */
    CloudCtl* ctl;              /* [nclouds] */
    int64_t total_tiles;        /* warp tiles (32 parcels) over all clouds */
    CloudK<P, V> one;           /* with one cloud: its descriptor, read from parameter space */
    int64_t wait_cycles = 0;    /* ring kernels: pipeline-wait limit in SM cycles, 0 = ~1 s;
                                   negative: the failure-detection test (ring_wait_limit) */
};

/* Unstructured tetrahedral mesh (st_tet.cu). */
struct TetMeshK {
    const double4* planes;      /* [nt][4] outward face planes (n0, n1, n2, c), s = n.x - c */
    const float4* planes32;     /* the same planes rounded to FP32 (the walk's pre-check) */
    float xmax;                 /* max |coordinate| of any point of the box, rounded up */
    int32_t pad0;
    const int32_t* nbr;         /* [nt][4] tet across the face opposite local vertex k, or -1 */
    int64_t nt;
    double origin[3];
    double ending[3];
    int32_t hop_limit;          /* face-walk hops per substep before a parcel counts as lost */
    int32_t pad;
};

template <class V>
struct TetStepArgs {
    TetMeshK mesh;
    PhysK<V> phys;
    double dtP;
    V dtV;
    V fscale;
    V fscale_lo;                         /* mixed precision: FP64 factor - fscale, else 0 */
    int32_t nclouds;
    const V* U;                          /* [nt*3] */
    const CloudK<double, V>* clouds;
    CloudCtl* ctl;
    int64_t total_tiles;                 /* warp tiles of WARP_TILE parcels */
    unsigned long long* hop_hist;        /* [8] walk lengths per substep, or nullptr */
    CloudK<double, V> one;               /* with one cloud: its descriptor (kernel parameters) */
    int64_t wait_cycles = 0;             /* ring kernel: pipeline-wait limit (as StepArgs) */
};

template <class V>
cudaError_t launch_step_tet(const TetStepArgs<V>& a, int dep, int grid, int block,
                            cudaStream_t s);
template <class V>
int step_tet_max_active_blocks(int dep, int block);
/* The tet step of a single cloud as a shared-memory ring (st_ring.cuh): true when it can run
 * this step (one cloud, a real deposit mode, 16-byte aligned arrays). */
template <class V>
bool tet_ring_eligible(const TetStepArgs<V>& a, int dep);
template <class V>
cudaError_t launch_step_tet_ring(const TetStepArgs<V>& a, int dep, int nsm, cudaStream_t s);
template <class V>
cudaError_t tet_ring_prepare();
/* Walks every parcel from hint[i] to the tet that contains it (hop limit of the mesh);
 * cells[i] = tet or -1, and `outside` counts failures. */
/* Face planes of every tet (canonical vertex order) from vertices and vertex ids. */
cudaError_t launch_tet_planes(const double* verts, const int32_t* tets, int64_t nt,
                              double4* planes, float4* planes32, cudaStream_t s);
cudaError_t launch_tet_locate(const TetMeshK& m, const double* x, const double* y,
                              const double* z, const int32_t* hint, int64_t n, int32_t* cells,
                              unsigned long long* outside, cudaStream_t s);

/* Arguments of the adjoint kernels (st_adjoint.cu). */
template <class P, class V>
struct AdjArgs {
    MeshK<P> mesh;
    PhysK<V> phys;
    P dtP;
    V dtV;
    int64_t n;                  /* parcels */
    int T;                      /* steps */
    int C;                      /* checkpoint interval */
    int limbs;                  /* fixed-point limbs of the mean source */
    const P* x;
    const P* y;
    const P* z;
    const V* u;
    const V* v;
    const V* w;
    const V* d;
    const V* U;                 /* [nCells*3] */
    const V* fs;                /* [T] fluid factor per step */
    const V* fs_lo;             /* [T] mixed precision: FP64 factor - fs, else zeros */
    unsigned long long* acc;    /* [ncomp*limbs] mean-source accumulator */
    CloudCtl* ctl;              /* scale and counters of the adjoint run */
    P* ck_x;                    /* checkpoints [nseg][3][n] */
    V* ck_v;
    V* rec_v;                   /* forward records of one segment [C][3][n] */
    int32_t* rec_c;             /* [C][n] */
    uint8_t* rec_b;             /* [C][n] */
    const double* G;            /* dJ/dS_n per cell component [ncomp] */
    V* adj_v;                   /* velocity cotangent [3][n] */
    double* partials;           /* [nseg][grid][2] parameter partials */
};

template <class P, class V>
cudaError_t launch_adj_forward(const AdjArgs<P, V>& a, bool probe, cudaStream_t s);
template <class P, class V>
cudaError_t launch_adj_reverse(const AdjArgs<P, V>& a, int seg, int len, int grid,
                               cudaStream_t s);
cudaError_t launch_adj_scale(CloudCtl* ctl, cudaStream_t s);
cudaError_t launch_adj_mean(const unsigned long long* acc, const CloudCtl* ctl, int limbs,
                            int T, double* mean, int64_t ncomp, cudaStream_t s);

/* Sets the thread-local message returned by st_last_error (st_abi.cu). */
void st_set_last_error(const char* msg);

/* Launchers implemented in st_kernels.cu (all asynchronous on `s`). */
template <class P, class V>
cudaError_t launch_step(const StepArgs<P, V>& a, int dep, int grid, int block, cudaStream_t s);
template <class P, class V>
int step_max_active_blocks(int dep, int block);
/* The step of a single cloud as a persistent shared-memory ring (st_ring.cu); deposits
 * DEP_DET1, DEP_DET2 or DEP_ATOMIC.  Every parcel array must be 16-byte aligned. */
template <class P, class V>
cudaError_t launch_step_ring(const StepArgs<P, V>& a, int dep, int nsm, cudaStream_t s);
/* Shared-memory opt-in of the ring kernels of a precision on the current device. */
template <class P, class V>
cudaError_t ring_prepare();
/* true when launch_step_ring can run this step */
template <class P, class V>
bool ring_eligible(const StepArgs<P, V>& a, int dep);

/* Fixed point -> FP64 source [nclouds][stride] (and, when src32 is not null, its FP32
 * rounding in the same layout), next scale per cloud. */
cudaError_t launch_finalize(int limbs, unsigned long long* acc, double* src, float* src32,
                            CloudCtl* ctl, const int32_t* Lsrc, unsigned int* counter,
                            int nclouds, int64_t stride, int grid_x, cudaStream_t s);
/* Scale of the step just run -> Lfin, next scale from its largest deposit (overlapped
 * finalize: the finalize then reads Lfin). */
cudaError_t launch_next_scale(CloudCtl* ctl, int32_t* Lfin, int nclouds, cudaStream_t s);
cudaError_t launch_set_scale(CloudCtl* ctl, int nclouds, cudaStream_t s);
cudaError_t launch_ctl_exponents(CloudCtl* ctl, int32_t* e, int nclouds, bool to_ctl,
                                 cudaStream_t s);
cudaError_t launch_zero_f64(double* p, int64_t n, cudaStream_t s);
cudaError_t launch_f64_to_f32(const double* in, float* out, int64_t n, cudaStream_t s);
cudaError_t launch_f32_to_f64(const float* in, double* out, int64_t n, cudaStream_t s);
template <class P, class V>
cudaError_t launch_init_cloud(uint64_t seed, int cloud, int nclouds, int64_t n,
                              const MeshK<P>& m, const double origin[3], const double ending[3],
                              double d_min, double d_max, P* x, P* y, P* z, V* u, V* v, V* w,
                              V* d, int32_t* id, cudaStream_t s);
cudaError_t launch_convert(const void* in, int in_bytes, void* out, int out_bytes, int64_t n,
                           cudaStream_t s);
cudaError_t launch_extrapolate(const double* s, double* est, float* est32, int64_t n,
                               cudaStream_t st);

/* Morton re-sort and order restoration (st_sort.cu). */
template <class P, class V>
struct SortBufs {
    P* x[2];
    P* y[2];
    P* z[2];
    V* u[2];
    V* v[2];
    V* w[2];
    V* d[2];
    int32_t* id[2];
    int32_t* cell[2];       /* tet meshes: owning tet, sorted along; nullptr on hex meshes */
    uint32_t* keys[2];
    uint32_t* perm[2];
    /* counting sort (key range of at most 2^COUNT_SORT_MAX_BITS): per-key counts and
     * offsets, shared by the clouds of a handle */
    uint32_t* bins;
    uint32_t* offsets;
    void* scan_temp;
    size_t scan_temp_bytes;
};
constexpr int COUNT_SORT_MAX_BITS = 24;
size_t count_sort_scan_bytes(int key_bits);
/* key_bits: bits of the (coarsened) key, at most COUNT_SORT_MAX_BITS; key_shift: low bits
 * dropped from each Morton coordinate, the linear cell index or the owning tet */
template <class P, class V>
cudaError_t sort_cloud(SortBufs<P, V>& b, int cur, int64_t n, const MeshK<P>& mesh, int key_bits,
                       int key_shift, bool morton, cudaStream_t s, int* launches);
template <class P, class V>
cudaError_t unpermute_cloud(SortBufs<P, V>& b, int cur, int64_t n, cudaStream_t s);
cudaError_t cells_unpermute(const int32_t* id, const int32_t* cell, int64_t n, int32_t* out,
                            cudaStream_t s);
/* State ([6][m] FP64) and owning cells of the parcels ids[0..m) (st_set_parcels indices,
 * each in [0, n)); uses b.perm[0] as scratch. */
template <class P, class V>
cudaError_t sample_cloud(SortBufs<P, V>& b, int cur, int64_t n, const MeshK<P>& mesh,
                         const int32_t* ids, int64_t m, double* out, int32_t* cells_out,
                         cudaStream_t s);
template <class P>
cudaError_t cells_cloud(const P* x, const P* y, const P* z, const int32_t* id, int64_t n,
                        const MeshK<P>& mesh, int32_t* cells_out, unsigned long long* outside,
                        cudaStream_t s);

}  // namespace st

#endif
