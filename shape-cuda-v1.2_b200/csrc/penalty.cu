// Model sums behind the objective's penalty terms (src/shape/penalties.c:
// 121-1236, src/shape/realize_mod.c:757-838): the uniform-density moments of
// the realized model (volume, first moment, inertia tensor; the facet
// integrals of src/shape/facmom.c), the sums over edges of the nonsmooth
// and concavity terms, and the sum and maximum of the squared vertex
// deviation lengths. The host turns these into each penalty.
//
// One pass over facets, edges and vertices by a grid of fixed shape writes
// per-block partials; a one-block kernel reduces them in a fixed order, so
// the sums are the same on every run. A model of several components first
// gets check_surface's active flags (src/shape/realize_mod.c:572-756), which
// leave the facets, edges and vertices inside another component out of
// the sums, as compute_moments and the penalties do.
#include <cuda_runtime.h>

#include "kernels.h"

namespace shape {

namespace {

constexpr int MS_THREADS = 256;
constexpr int MS_BLOCKS = 148;

__device__ __forceinline__ double d3(const double4 &a, const double4 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__device__ __forceinline__ double comp(const double4 &p, int k) { return k == 0 ? p.x : (k == 1 ? p.y : p.z); }

// check_surface's tolerances (src/shape/realize_mod.c:142-144): the edge
// tolerance of the ray-facet test, the distance tolerance of an
// intersection beyond the point and of two edge crossings being one, and
// the edge crossings one ray may record.
constexpr double SURF_EDGETOL = 1.0e-14;
constexpr double SURF_RTOL = 1000 * 1.0e-14;
constexpr int SURF_MAXEDGE = 100;

// Where the ray r * u from the origin meets the plane of facet (v0, v1, v2)
// with normal n (Badouel's projection method, as src/shape/rayfacint.c
// states it, with the same operations): r along the ray, (s, t) in the facet
// (v0 + s (v1 - v0) + t (v2 - v1)); true when the point lies in the facet
// to within tol.
__device__ bool ray_facet(const double u[3], const double4 &v0, const double4 &v1, const double4 &v2,
                          const double4 &n, double tol, double &r, double &s, double &t)
{
    const double a[3] = {0.0, 0.0, 0.0};
    const double p0[3] = {v0.x, v0.y, v0.z}, p1[3] = {v1.x, v1.y, v1.z}, p2[3] = {v2.x, v2.y, v2.z};
    const double nn[3] = {n.x, n.y, n.z};
    double ra0[3], r01[3], r12[3], r0p[3];
    for (int i = 0; i < 3; i++) {
        ra0[i] = p0[i] - a[i];
        r01[i] = p1[i] - p0[i];
        r12[i] = p2[i] - p1[i];
    }
    const double ndu = nn[0] * u[0] + nn[1] * u[1] + nn[2] * u[2];
    if (ndu == 0.0) {
        r = s = t = -SHAPE_HUGENUMBER;
        return false;
    }
    r = (nn[0] * ra0[0] + nn[1] * ra0[1] + nn[2] * ra0[2]) / ndu;
    for (int i = 0; i < 3; i++) r0p[i] = (a[i] + r * u[i]) - p0[i];
    const double ax = fabs(nn[0]), ay = fabs(nn[1]), az = fabs(nn[2]);
    int i0 = 0;
    double mx = ax;
    if (ay > mx) { i0 = 1; mx = ay; }
    if (az > mx) i0 = 2;
    const int i1 = (i0 + 1) % 3, i2 = (i1 + 1) % 3;
    if (r01[i1] == 0.0) {
        t = r0p[i1] / r12[i1];
        s = (r0p[i2] - t * r12[i2]) / r01[i2];
    } else {
        t = (r0p[i2] * r01[i1] - r0p[i1] * r01[i2]) / (r12[i2] * r01[i1] - r12[i1] * r01[i2]);
        s = (r0p[i1] - t * r12[i1]) / r01[i1];
    }
    return (s >= -tol) && (s <= 1.0 + tol) && (t >= -tol) && (t <= s + tol);
}

// check_surface for a model of several components: one thread per vertex
// (the ray from the origin through it) and per facet (through its
// centroid). The point is inactive when, for some other component, the ray
// crosses that component's surface an odd number of times beyond the point;
// crossings at a facet edge or corner are counted once per distinct
// distance. Components are tried in the reference's order (0 or 1 first,
// skipping the point's own), stopping at the first that encloses it.
__global__ void __launch_bounds__(MS_THREADS) k_check_surface(ModelSumArgs a)
{
    const ModelDev &m = a.m;
    const int idx = blockIdx.x * MS_THREADS + threadIdx.x;
    if (idx >= m.nv + m.nf) return;
    const bool isv = idx < m.nv;
    double u[3];
    int c;
    if (isv) {
        const double4 p = m.vx[idx];
        u[0] = p.x; u[1] = p.y; u[2] = p.z;
        c = m.vcomp[idx];
    } else {
        const int f = idx - m.nv;
        const double4 p0 = m.vx[m.fv[3 * f]], p1 = m.vx[m.fv[3 * f + 1]], p2 = m.vx[m.fv[3 * f + 2]];
        u[0] = (p0.x + p1.x + p2.x) / 3;
        u[1] = (p0.y + p1.y + p2.y) / 3;
        u[2] = (p0.z + p1.z + p2.z) / 3;
        c = m.vcomp[m.fv[3 * f]];
    }
    double dist = 0.0;
    dist += u[0] * u[0];
    dist += u[1] * u[1];
    dist += u[2] * u[2];
    dist = sqrt(dist);
    if (dist != 0.0)
        for (int i = 0; i < 3; i++) u[i] /= dist;
    double r_edge[SURF_MAXEDGE];
    bool act = true;
    int c2 = (c == 0) ? 1 : 0;
    do {
        const int2 fr = a.comp_facets[c2];
        int nint = 0, nedge = 0;
        for (int f2 = fr.x; f2 < fr.x + fr.y; f2++) {
            double r, s, t;
            if (!ray_facet(u, m.vx[m.fv[3 * f2]], m.vx[m.fv[3 * f2 + 1]], m.vx[m.fv[3 * f2 + 2]], m.fn[f2],
                           SURF_EDGETOL, r, s, t))
                continue;
            if (!(r > dist + SURF_RTOL)) continue;
            if (fabs(s) < SURF_EDGETOL || fabs(s - 1.0) < SURF_EDGETOL || fabs(t) < SURF_EDGETOL ||
                fabs(t - s) < SURF_EDGETOL) {
                bool fresh = true;
                for (int k = 0; k < nedge; k++)
                    if (fabs(r - r_edge[k]) < SURF_RTOL) fresh = false;
                if (fresh) {
                    if (nedge == SURF_MAXEDGE) {
                        atomicExch(a.surf_err, 1);
                        break;
                    }
                    r_edge[nedge++] = r;
                    nint++;
                }
            } else {
                nint++;
            }
        }
        if (nint % 2 == 1) act = false;
        c2 = (c2 == c - 1) ? c2 + 2 : c2 + 1;
    } while (act && c2 < a.ncomp);
    if (isv) a.act_v[idx] = act ? 1 : 0;
    else a.act_f[idx - m.nv] = act ? 1 : 0;
}

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
        if (!a.act_f || a.act_f[f])
            facet_moments(m.vx[m.fv[3 * f]], m.vx[m.fv[3 * f + 1]], m.vx[m.fv[3 * f + 2]], m.fn[f], acc);
    // edges (v1, v3, f1, f2): v3 is f1's vertex off the edge, v1 an end;
    // an edge is active when both its ends are
    for (int s = t0; s < a.nsides; s += stride) {
        const int4 e = a.sides[s];
        if (a.act_v && !(a.act_v[e.x] && a.act_v[a.side_v2[s]])) continue;
        acc[MSUM_NSIDES] += 1.0;
        const double4 n1 = m.fn[e.z], n2 = m.fn[e.w];
        const double x = 1.0 - d3(n1, n2);
        acc[MSUM_NONSMOOTH] += x * x * x * x;
        const double4 p1 = m.vx[e.x], p3 = m.vx[e.y];
        const double4 disp = make_double4(p3.x - p1.x, p3.y - p1.y, p3.z - p1.z, 0.0);
        if (d3(disp, n2) > 0.0) acc[MSUM_CONCAVITY] += x * x;
    }
    // vertex deviation lengths |u . scale| * r (the vertex's component's
    // scale factors)
    for (int v = t0; v < m.nv; v += stride) {
        if (a.act_v && !a.act_v[v]) continue;
        acc[MSUM_NVERT] += 1.0;
        const double *sc = m.scale + (m.vcomp ? 3 * m.vcomp[v] : 0);
        double len = 0.0;
        for (int j = 0; j < 3; j++) {
            const double y = m.u[3 * v + j] * sc[j];
            len += y * y;
        }
        const double d = sqrt(len) * m.r[v];
        acc[MSUM_RDEV] += d * d;
        acc[MSUM_RDEV_MAX] = fmax(acc[MSUM_RDEV_MAX], d * d);
    }
    if (t0 == 0 && a.surf_err) acc[MSUM_SURF_ERR] = (double)*a.surf_err;
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

void launch_check_surface(const ModelSumArgs &a, cudaStream_t s)
{
    const int n = a.m.nv + a.m.nf;
    k_check_surface<<<(n + MS_THREADS - 1) / MS_THREADS, MS_THREADS, 0, s>>>(a);
}

void launch_model_sums(const ModelSumArgs &a, cudaStream_t s)
{
    const size_t smem = sizeof(double) * MSUM_N * MS_THREADS;
    k_model_sums<<<MS_BLOCKS, MS_THREADS, smem, s>>>(a);
    k_model_sums_final<<<1, MS_THREADS, smem, s>>>(a, MS_BLOCKS);
}

}  // namespace shape
