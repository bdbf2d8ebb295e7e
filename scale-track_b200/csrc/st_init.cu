/*
 * st_init.cu -- parcels generated on the device (st_init_parcels): one thread per parcel
 * evaluates the counter-based Hilbert-clustered generator of st_init.h, so a cloud of any
 * size is created without a host round trip.
 */
#include <cstdint>
#include <cuda_runtime.h>

#include "st_internal.h"
#include "st_init.h"

namespace st {

template <class P, class V>
__global__ void k_init_cloud(uint64_t seed, int cloud, int nclouds, int64_t n, MeshK<P> m,
                             double o0, double o1, double o2, double e0, double e1, double e2,
                             double d_min, double d_max, P* __restrict__ x, P* __restrict__ y,
                             P* __restrict__ z, V* __restrict__ u, V* __restrict__ v,
                             V* __restrict__ w, V* __restrict__ d, int32_t* __restrict__ id)
{
    const double origin[3] = {o0, o1, o2};
    const double ending[3] = {e0, e1, e2};
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n;
         j += (int64_t)gridDim.x * blockDim.x) {
        P xyz[3];
        double dd;
        st_init_parcel<P>(seed, cloud, nclouds, (uint64_t)j, m.N, origin, ending, xyz, dd, d_min,
                          d_max);
        x[j] = xyz[0];
        y[j] = xyz[1];
        z[j] = xyz[2];
        u[j] = (V)0;
        v[j] = (V)0;
        w[j] = (V)0;
        d[j] = (V)dd;
        id[j] = (int32_t)j;
    }
}

template <class P, class V>
cudaError_t launch_init_cloud(uint64_t seed, int cloud, int nclouds, int64_t n,
                              const MeshK<P>& m, const double origin[3], const double ending[3],
                              double d_min, double d_max, P* x, P* y, P* z, V* u, V* v, V* w,
                              V* d, int32_t* id, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    int64_t g = (n + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_init_cloud<P, V><<<(int)g, 256, 0, s>>>(seed, cloud, nclouds, n, m, origin[0], origin[1],
                                              origin[2], ending[0], ending[1], ending[2], d_min,
                                              d_max, x, y, z, u, v, w, d, id);
    return cudaGetLastError();
}

template cudaError_t launch_init_cloud<float, float>(uint64_t, int, int, int64_t,
                                                     const MeshK<float>&, const double*,
                                                     const double*, double, double, float*,
                                                     float*, float*, float*, float*, float*,
                                                     float*, int32_t*, cudaStream_t);
template cudaError_t launch_init_cloud<double, float>(uint64_t, int, int, int64_t,
                                                      const MeshK<double>&, const double*,
                                                      const double*, double, double, double*,
                                                      double*, double*, float*, float*, float*,
                                                      float*, int32_t*, cudaStream_t);
template cudaError_t launch_init_cloud<double, double>(uint64_t, int, int, int64_t,
                                                       const MeshK<double>&, const double*,
                                                       const double*, double, double, double*,
                                                       double*, double*, double*, double*,
                                                       double*, double*, int32_t*, cudaStream_t);

}  // namespace st
