// Model sums behind the objective's penalty terms (src/shape/penalties.c:
// 121-1236, src/shape/realize_mod.c:757-838): the uniform-density moments of
// the realized model (volume, first moment, inertia tensor; the facet
// integrals of src/shape/facmom.c), the sums over edges of the nonsmooth
// and concavity terms, and the sum and maximum of the squared vertex
// deviation lengths. The host turns these into each penalty.
//
// One pass over facets, edges and vertices by a grid of fixed shape writes
// per-block partials; a one-block kernel reduces them in a fixed order, so
// the sums are the same on every run.
#include <cuda_runtime.h>

#include "kernels.h"

namespace shape {

namespace {

constexpr int MS_THREADS = 256;
constexpr int MS_BLOCKS = 148;

__device__ __forceinline__ double d3(const double4 &a, const double4 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ double comp(const double4 &p, int k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }

// Moments of the prism between facet (p0, p1, p2), normal n, and the
// coordinate plane normal to axis k, projected along k, for each k in the
// cyclic order z, y, x: first moment along k, -integral of (b * k) with b
// the axis after k, and integral of k^2 (exact integrals over the prism).
// The volume is the z-projection's.
__device__ void facet_moments(const double4 &p0, const double4 &p1, const double4 &p2, const double4 &n,
                              double acc[MSUM_N])
{
    const int order[3] = {2, 1, 0};
    double first[3], cross[3], sq[3];
    for (int i = 0; i < 3; i++) {
        const int k = order[i], a = (k + 1) % 3, b = (k + 2) % 3;
        const double a0 = comp(p0, a), a1 = comp(p1, a), a2 = comp(p2, a);
        const double b0 = comp(p0, b), b1 = comp(p1, b), b2 = comp(p2, b);
        const double z0 = comp(p0, k), z1 = comp(p1, k), z2 = comp(p2, k);
        const double jac = fabs((a1 - a0) * (b2 - b1) - (a2 - a1) * (b1 - b0));
        const double sj = comp(n, k) < 0.0 ? -jac : jac;
        const double zs = z0 + z1 + z2, zq = z0 * z0 + z1 * z1 + z2 * z2;
        if (i == 0) acc[MSUM_VOLUME] += sj * zs / 6.0;
        first[k] = sj * (z0 * zs + z1 * (z1 + z2) + z2 * z2) / 24.0;
        cross[k] = -(sj / 120.0) * ((b0 + b1 + b2) * zq + 2.0 * (b0 * z0 + b1 * z1 + b2 * z2) * zs +
                                    (b0 * z1 * z2 + b1 * z0 * z2 + b2 * z0 * z1));
        sq[k] = (sj / 60.0) * (zq * zs + z0 * z1 * z2);
    }
    acc[MSUM_COM + 0] += first[0];
    acc[MSUM_COM + 1] += first[1];
    acc[MSUM_COM + 2] += first[2];
    acc[MSUM_IXX] += sq[2] + sq[1];
    acc[MSUM_IYY] += sq[2] + sq[0];
    acc[MSUM_IZZ] += sq[1] + sq[0];
    acc[MSUM_IXY] += cross[1];
    acc[MSUM_IXZ] += cross[0];
    acc[MSUM_IYZ] += cross[2];
}

// Block reduction of MSUM_N values (sums, and a maximum for MSUM_RDEV_MAX)
// in a fixed tree order; thread 0 ends with the result.
__device__ void block_reduce(double acc[MSUM_N], double *sh)
{
    for (int q = 0; q < MSUM_N; q++) sh[q * MS_THREADS + threadIdx.x] = acc[q];
    __syncthreads();
    for (int w = MS_THREADS / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int q = 0; q < MSUM_N; q++) {
                double &x = sh[q * MS_THREADS + threadIdx.x];
                const double y = sh[q * MS_THREADS + threadIdx.x + w];
                x = (q == MSUM_RDEV_MAX) ? fmax(x, y) : x + y;
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < MSUM_N; q++) acc[q] = sh[q * MS_THREADS];
}

__global__ void __launch_bounds__(MS_THREADS) k_model_sums(ModelSumArgs a)
{
    extern __shared__ double sh[];
    double acc[MSUM_N];
    for (int q = 0; q < MSUM_N; q++) acc[q] = 0.0;
    const ModelDev &m = a.m;
    const int stride = gridDim.x * MS_THREADS, t0 = blockIdx.x * MS_THREADS + threadIdx.x;
    for (int f = t0; f < m.nf; f += stride)
        facet_moments(m.vx[m.fv[3 * f]], m.vx[m.fv[3 * f + 1]], m.vx[m.fv[3 * f + 2]], m.fn[f], acc);
    // edges (v1, v3, f1, f2): v3 is f1's vertex off the edge, v1 an end
    for (int s = t0; s < a.nsides; s += stride) {
        const int4 e = a.sides[s];
        const double4 n1 = m.fn[e.z], n2 = m.fn[e.w];
        const double x = 1.0 - d3(n1, n2);
        acc[MSUM_NONSMOOTH] += x * x * x * x;
        const double4 p1 = m.vx[e.x], p3 = m.vx[e.y];
        const double4 disp = make_double4(p3.x - p1.x, p3.y - p1.y, p3.z - p1.z, 0.0);
        if (d3(disp, n2) > 0.0) acc[MSUM_CONCAVITY] += x * x;
    }
    // vertex deviation lengths |u . scale| * r
    for (int v = t0; v < m.nv; v += stride) {
        double len = 0.0;
        for (int j = 0; j < 3; j++) {
            const double y = m.u[3 * v + j] * m.scale[j];
            len += y * y;
        }
        const double d = sqrt(len) * m.r[v];
        acc[MSUM_RDEV] += d * d;
        acc[MSUM_RDEV_MAX] = fmax(acc[MSUM_RDEV_MAX], d * d);
    }
    block_reduce(acc, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < MSUM_N; q++) a.part[(size_t)blockIdx.x * MSUM_N + q] = acc[q];
}

__global__ void __launch_bounds__(MS_THREADS) k_model_sums_final(ModelSumArgs a, int nblocks)
{
    extern __shared__ double sh[];
    double acc[MSUM_N];
    for (int q = 0; q < MSUM_N; q++) acc[q] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += MS_THREADS)
        for (int q = 0; q < MSUM_N; q++) {
            const double y = a.part[(size_t)b * MSUM_N + q];
            acc[q] = (q == MSUM_RDEV_MAX) ? fmax(acc[q], y) : acc[q] + y;
        }
    block_reduce(acc, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < MSUM_N; q++) a.out[q] = acc[q];
}

}  // namespace

int model_sums_blocks() { return MS_BLOCKS; }

void launch_model_sums(const ModelSumArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double) * MSUM_N * MS_THREADS;
    k_model_sums<<<MS_BLOCKS, MS_THREADS, smem, s>>>(a);
    k_model_sums_final<<<1, MS_THREADS, smem, s>>>(a, MS_BLOCKS);
}

}  // namespace shape
