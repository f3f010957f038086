// Tile rasterizer with fused delay-Doppler synthesis (templated on the
// arithmetic type T; included by raster_f64.cu, compiled without FMA
// contraction, and raster_f32.cu).
//
// One CTA owns one 16x16 tile of one POS view; each thread owns one pixel.
// The tile's facet bin (filled by k_bin) is loaded into shared memory and
// sorted by facet index, then facets are staged 128 at a time and every
// pixel replays them IN INDEX ORDER with posvis's update rule
// (src/shape/posvis.c:205-292): a facet takes a pixel when z > zz or the
// pixel is still blank, cos(e) (and cos(i)) change only when the smoothed
// normal faces the observer. Replaying in index order per pixel reproduces
// the sequential reference exactly: exact-z ties keep the lower facet and
// limb pixels inherit cos(e) from the earlier winner, as on the CPU. No
// atomics are needed for the z-buffer because a pixel has a single owner.
//
// For radar views the pixel then computes its pos2deldop contributions
// (src/shape/pos2deldop.c:305-535) and scatter-adds them into the frame's
// fit image, so POS maps never travel through HBM unless requested.
#pragma once

#include <climits>

#include "kernels.h"

namespace shape {

template <typename T> struct Vec4;
template <> struct Vec4<double> { using type = double4; };
template <> struct Vec4<float> { using type = float4; };

template <typename T>
struct Stage {
    T v00, v01, v02, A, B, C, D, E, F, den;
    T nx, ny, nz;
    int i1, i2, j1, j2;
    int f, c0, c1, c2;
};

template <typename T> __device__ inline T tsin(T x);
template <> __device__ inline double tsin<double>(double x) { return sin(x); }
template <> __device__ inline float tsin<float>(float x) { return sinf(x); }
template <typename T> __device__ inline T tpow(T x, T y);
template <> __device__ inline double tpow<double>(double x, double y) { return pow(x, y); }
template <> __device__ inline float tpow<float>(float x, float y) { return powf(x, y); }
template <typename T> __device__ inline T texp(T x);
template <> __device__ inline double texp<double>(double x) { return exp(x); }
template <> __device__ inline float texp<float>(float x) { return expf(x); }

// SINC2 / TRI / TRI2 macros (src/macros/func.h:6-8)
template <typename T> __device__ inline T sinc2(T x)
{
    T tmp = fabs((T)3.141592653589793 * x);
    if (tmp > (T)1.0e-4) {
        tmp = tsin<T>(tmp) / tmp;
        return tmp * tmp;
    }
    return (T)1.0;
}
template <typename T> __device__ inline T tri(T x) { T t = (T)1 - fabs(x); return t > (T)0 ? t : (T)0; }
template <typename T> __device__ inline T tri2(T x) { T t = (T)1 - fabs(x); return t > (T)0 ? t * t : (T)0; }

// radlaw for the facet-independent laws (src/shape/radlaw.c:44-148)
template <typename T> __device__ T radlaw_dev(const RadarLawDev &L, T c)
{
    T v = (T)-9.99, tan2inc, sin2inc, arg;
    switch (L.type) {
    case SHAPE_RADLAW_COSINE_DIFF:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * tpow<T>(c, 2 * (T)L.diff_C - 1);
        break;
    case SHAPE_RADLAW_GAUSSIAN:
        if (c >= (T)L.qs_cos_cutoff) {
            tan2inc = 1 / (c * c) - 1;
            v = (T)L.qs_R * (T)L.qs_C * texp<T>(-(T)L.qs_C * tan2inc) / (c * c * c * c * c);
        } else v = 0;
        break;
    case SHAPE_RADLAW_HAGFORS:
        if (c >= (T)L.qs_cos_cutoff) {
            sin2inc = 1 - c * c;
            arg = c * c * c * c + (T)L.qs_C * sin2inc;
            v = (T)0.5 * (T)L.qs_R * (T)L.qs_C * tpow<T>(arg, (T)-1.5) / c;
        } else v = 0;
        break;
    case SHAPE_RADLAW_COSINE_QS:
        if (c >= (T)L.qs_cos_cutoff)
            v = (T)L.qs_R * ((T)L.qs_C + 1) * tpow<T>(c, 2 * (T)L.qs_C - 1);
        else v = 0;
        break;
    case SHAPE_RADLAW_GAUSSIAN_COSINE:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * tpow<T>(c, 2 * (T)L.diff_C - 1);
        if (c >= (T)L.qs_cos_cutoff) {
            tan2inc = 1 / (c * c) - 1;
            v += (T)L.qs_R * (T)L.qs_C * texp<T>(-(T)L.qs_C * tan2inc) / (c * c * c * c * c);
        }
        break;
    case SHAPE_RADLAW_HAGFORS_COSINE:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * tpow<T>(c, 2 * (T)L.diff_C - 1);
        if (c >= (T)L.qs_cos_cutoff) {
            sin2inc = 1 - c * c;
            arg = c * c * c * c + (T)L.qs_C * sin2inc;
            v += (T)0.5 * (T)L.qs_R * (T)L.qs_C * tpow<T>(arg, (T)-1.5) / c;
        }
        break;
    case SHAPE_RADLAW_COSINE_COSINE:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * tpow<T>(c, 2 * (T)L.diff_C - 1);
        if (c >= (T)L.qs_cos_cutoff)
            v += (T)L.qs_R * ((T)L.qs_C + 1) * tpow<T>(c, 2 * (T)L.qs_C - 1);
        break;
    default:
        break;
    }
    return v;
}

// Stage one facet for a view: culling, bbox and the per-facet terms of the
// s, t, z expressions (src/shape/posvis.c:146-223). Returns false when the
// facet faces away or misses the tile [ti0, ti1] x [tj0, tj1].
template <typename T>
__device__ bool stage_facet(const RasterArgs &a, const FrameGeom &g, int f,
                            int ti0, int ti1, int tj0, int tj1, Stage<T> &s)
{
    using T4 = typename Vec4<T>::type;
    const T4 *vt = static_cast<const T4 *>(a.vt) + g.vt_base;
    double4 nb = a.fn[f];
    double nn[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        nn[r] = 0.0;
        nn[r] += g.oa[3 * r + 0] * nb.x;
        nn[r] += g.oa[3 * r + 1] * nb.y;
        nn[r] += g.oa[3 * r + 2] * nb.z;
    }
    if (!(nn[2] > 0.0)) return false;
    int4 c = a.fvi[f];
    T4 p0 = vt[c.x], p1 = vt[c.y], p2 = vt[c.z];
    const double kmpp = g.kmpp;
    const int n = g.n;
    double x0d = p0.x, x1d = p1.x, x2d = p2.x, y0d = p0.y, y1d = p1.y, y2d = p2.y;
    double xmin = (x0d < ((x1d < x2d) ? x1d : x2d)) ? x0d : ((x1d < x2d) ? x1d : x2d);
    double xmax = (x0d > ((x1d > x2d) ? x1d : x2d)) ? x0d : ((x1d > x2d) ? x1d : x2d);
    double ymin = (y0d < ((y1d < y2d) ? y1d : y2d)) ? y0d : ((y1d < y2d) ? y1d : y2d);
    double ymax = (y0d > ((y1d > y2d) ? y1d : y2d)) ? y0d : ((y1d > y2d) ? y1d : y2d);
    double imin_d = floor(xmin / kmpp - SHAPE_SMALLVAL + 0.5);
    double imax_d = floor(xmax / kmpp + SHAPE_SMALLVAL + 0.5);
    double jmin_d = floor(ymin / kmpp - SHAPE_SMALLVAL + 0.5);
    double jmax_d = floor(ymax / kmpp + SHAPE_SMALLVAL + 0.5);
    int imin = (imin_d < (double)INT_MIN) ? INT_MIN : (int)imin_d;
    int imax = (imax_d > (double)INT_MAX) ? INT_MAX : (int)imax_d;
    int jmin = (jmin_d < (double)INT_MIN) ? INT_MIN : (int)jmin_d;
    int jmax = (jmax_d > (double)INT_MAX) ? INT_MAX : (int)jmax_d;
    int i1 = max(imin, -n), i2 = min(imax, n), j1 = max(jmin, -n), j2 = min(jmax, n);
    if (i1 > n || i2 < -n || j1 > n || j2 < -n) return false;
    if (i2 < ti0 || i1 > ti1 || j2 < tj0 || j1 > tj1) return false;
    s.v00 = p0.x; s.v01 = p0.y; s.v02 = p0.z;
    s.A = p2.y - p1.y;
    s.B = p2.x - p1.x;
    s.C = p1.x - p0.x;
    s.D = p1.y - p0.y;
    s.E = p1.z - p0.z;
    s.F = p2.z - p1.z;
    s.den = (T)1 / (s.C * s.A - s.B * s.D);
    s.nx = (T)nn[0]; s.ny = (T)nn[1]; s.nz = (T)nn[2];
    s.i1 = i1; s.i2 = i2; s.j1 = j1; s.j2 = j2;
    s.f = f; s.c0 = c.x; s.c1 = c.y; s.c2 = c.z;
    return true;
}

template <typename T> __device__ inline void atomic_add_fit(T *p, T v);
template <> __device__ inline void atomic_add_fit<double>(double *p, double v) { atomicAdd(p, v); }
template <> __device__ inline void atomic_add_fit<float>(float *p, float v) { atomicAdd(p, v); }

struct PixLimits {
    int idmin, idmax, ipmin, ipmax;
    double dmin, dmax, pmin, pmax;
};

// Delay / Doppler position and footprint of one lit POS pixel
// (src/shape/pos2deldop.c:318-367).
template <typename T>
struct PixDD {
    T delPOS, dopPOS, codefactor;
    int idel_min, idel_max, idop_min, idop_max;
    bool ok;   // in_bounds: the whole footprint lies inside the frame
};

template <typename T>
__device__ PixDD<T> pixel_dd_setup(const FrameGeom &g, int x, int y, T z, PixLimits &lim)
{
    PixDD<T> d;
    d.delPOS = z * (T)g.delfact + (T)g.delshift;
    const T const1 = (T)g.const1;
    d.idel_min = (int)floor(d.delPOS - const1) + 1;
    d.idel_max = (int)ceil(d.delPOS + const1) - 1;
    d.dopPOS = (T)g.ax * (T)x + (T)g.ay * (T)y + (T)g.dopshift;
    const T dopdiff_max = (T)g.dopdiff_max;
    const T half_w = (T)(g.sinc2width / 2.0);
    d.idop_min = (int)floor(d.dopPOS - dopdiff_max + 1 - half_w);
    d.idop_max = (int)floor(d.dopPOS + dopdiff_max + half_w);
    d.codefactor = (g.codemethod == SHAPE_CODE_SHORT)
                       ? sinc2<T>((d.dopPOS - (T)g.dopDC_vig) / (T)g.dopfftlen) : (T)1;
    lim.idmin = min(lim.idmin, d.idel_min);
    lim.idmax = max(lim.idmax, d.idel_max);
    lim.ipmin = min(lim.ipmin, d.idop_min);
    lim.ipmax = max(lim.ipmax, d.idop_max);
    lim.dmin = fmin(lim.dmin, (double)d.delPOS);
    lim.dmax = fmax(lim.dmax, (double)d.delPOS);
    lim.pmin = fmin(lim.pmin, (double)d.dopPOS);
    lim.pmax = fmax(lim.pmax, (double)d.dopPOS);
    d.ok = (d.idel_min >= 1) && (d.idel_max <= g.ndel) && (d.idop_min >= 1) && (d.idop_max <= g.ndop) &&
           (d.idel_max - d.idel_min + 1 <= SHAPE_MAXBINS);
    return d;
}

template <typename T> __device__ inline void atomic_add_any(T *p, T v) { atomicAdd(p, v); }

// Delay and Doppler response of one pixel and its scatter into `dst`, an
// image whose element (idel, idop) lives at dst[(idel - row0) * stride +
// (idop - col0)] (src/shape/pos2deldop.c:371-496). dst is either the frame's
// fit image in HBM or the tile's shared-memory accumulator.
template <typename T>
__device__ void pixel_dd_scatter(const RasterArgs &a, const FrameGeom &g, T cose, const PixDD<T> &d,
                                 T *dst, int row0, int col0, int stride)
{
    const T delPOS = d.delPOS, dopPOS = d.dopPOS, const1 = (T)g.const1;
    const int idel_min = d.idel_min, idel_max = d.idel_max, idop_min = d.idop_min, idop_max = d.idop_max;
    T del_c[SHAPE_MAXBINS];
    T dop_c[SHAPE_MAXBINS + 1];
    const int spb = g.spb;
    for (int idel = idel_min; idel <= idel_max; idel++) {
        T dc;
        if (g.codemethod != SHAPE_CODE_LONG_ORIG) {
            if (spb == 1) {
                dc = tri2<T>(delPOS - (T)idel);
            } else if (spb == 2) {
                T arg = (delPOS - ((T)idel - (T)g.const2)) / (T)g.spb_over_stride;
                dc = tri<T>(arg) + tri<T>(arg - (T)0.5);
                dc *= dc / 4;
            } else {
                dc = 0;
                int m_min = max((int)floor((delPOS - (T)idel - (T)g.const2) * (T)g.stride), 0);
                int m_max = min((int)ceil((delPOS - (T)idel + const1) * (T)g.stride), spb) - 1;
                T arg = (delPOS - ((T)idel - (T)g.const2)) / (T)g.spb_over_stride
                        - (T)m_min * (T)g.one_over_spb;
                for (int m = m_min; m <= m_max; m++) {
                    dc += tri<T>(arg);
                    arg -= (T)g.one_over_spb;
                }
                dc *= dc / (T)g.spb_sq;
            }
        } else {
            dc = tri2<T>((delPOS - (T)idel) / (T)g.spb_over_stride);
        }
        del_c[idel - idel_min] = dc;
    }
    const int nsinc2 = g.nsinc2;
    for (int idop = idop_min; idop <= idop_max; idop++) {
        T sm;
        if (nsinc2 == 1) {
            sm = sinc2<T>(dopPOS - (T)idop);
        } else if (nsinc2 == 2) {
            T bl = dopPOS + (T)g.dopdiff_bl - (T)idop;
            sm = (sinc2<T>(bl) + sinc2<T>(bl + (T)g.xincr) + sinc2<T>(bl + (T)g.yincr) +
                  sinc2<T>(bl + (T)g.xincr + (T)g.yincr)) / 4;
        } else {
            T left = dopPOS + (T)g.dopdiff_bl - (T)idop;
            sm = 0;
            for (int i = 0; i < nsinc2; i++) {
                T arg = left;
                for (int j = 0; j < nsinc2; j++) {
                    sm += sinc2<T>(arg);
                    arg += (T)g.xincr;
                }
                left += (T)g.yincr;
            }
            sm /= (T)g.nsinc2_sq;
        }
        dop_c[min(idop - idop_min, SHAPE_MAXBINS)] = sm;
    }
    T sumweights = 0;
    for (int idel = idel_min; idel <= idel_max; idel++)
        for (int idop = idop_min; idop <= idop_max; idop++)
            sumweights += del_c[idel - idel_min] * dop_c[min(idop - idop_min, SHAPE_MAXBINS)];
    const T kmpp = (T)g.kmpp;
    T amp = radlaw_dev<T>(a.laws[g.law], cose) * kmpp * kmpp * d.codefactor / sumweights;
    for (int idel = idel_min; idel <= idel_max; idel++) {
        T ad = amp * del_c[idel - idel_min];
        T *row = dst + (long long)(idel - row0) * stride - col0;
        for (int idop = idop_min; idop <= idop_max; idop++)
            atomic_add_any<T>(row + idop, ad * dop_c[min(idop - idop_min, SHAPE_MAXBINS)]);
    }
}

__device__ inline int warp_min(int v)
{
    for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline int warp_max(int v)
{
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline double warp_dmin(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ inline double warp_dmax(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <typename T>
__global__ void __launch_bounds__(RASTER_THREADS) k_raster(RasterArgs a)
{
    extern __shared__ __align__(16) unsigned char smem[];
    int *raw = reinterpret_cast<int *>(smem);
    int *ids = raw + a.cap;
    Stage<T> *st = reinterpret_cast<Stage<T> *>(smem + (((size_t)2 * a.cap * sizeof(int) + 15) & ~(size_t)15));
    __shared__ int s_nst;
    __shared__ int s_red[RASTER_THREADS / 32][4];
    __shared__ double s_redd[RASTER_THREADS / 32][4];
    __shared__ int s_redl[RASTER_THREADS / 32][4];
    __shared__ int s_box[RASTER_THREADS / 32][4];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

    for (int w = blockIdx.x; w < a.nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const FrameGeom &g = a.geoms[item.x];
        const int tile = item.y;
        const int tx = tile / g.tiles_x, ty = tile % g.tiles_x;
        const int n = g.n;
        const int ti0 = -n + tx * TILE_W, tj0 = -n + ty * TILE_W;
        const int ti1 = min(ti0 + TILE_W - 1, n), tj1 = min(tj0 + TILE_W - 1, n);
        const int pi = ti0 + tid / TILE_W, pj = tj0 + tid % TILE_W;
        const bool inframe = (pi <= n) && (pj <= n);
        const int count = a.bin_count[g.tile_base + tile];
        const bool writes_pos = (g.kind != VIEW_RADAR) || a.keep_pos;
        if (count == 0 && !writes_pos) continue;

        const T x0 = (T)pi * (T)g.kmpp, x1 = (T)pj * (T)g.kmpp;
        T zz = (T)(-SHAPE_HUGENUMBER), cosa = 0, cosb = 0;
        int fac = -1;
        const bool smooth = g.smooth != 0;
        const bool bistatic_obs = (g.kind == VIEW_LC_OBS);
        T oa[9];
#pragma unroll
        for (int k = 0; k < 9; k++) oa[k] = (T)g.oa[k];
        const T us0 = (T)g.usrc[0], us1 = (T)g.usrc[1], us2 = (T)g.usrc[2];

        auto replay = [&](int nst) {
            for (int k = 0; k < nst; k++) {
                const Stage<T> &s = st[k];
                if (pi < s.i1 || pi > s.i2 || pj < s.j1 || pj > s.j2) continue;
                const T dx = x0 - s.v00, dy = x1 - s.v01;
                const T sv = (dx * s.A - s.B * dy) * s.den;
                if (!((sv >= (T)-SHAPE_SMALLVAL) && (sv <= (T)1.0 + (T)SHAPE_SMALLVAL))) continue;
                const T tv = (s.C * dy - dx * s.D) * s.den;
                if (!((tv >= (T)-SHAPE_SMALLVAL) && (tv <= sv + (T)SHAPE_SMALLVAL))) continue;
                const T z = s.v02 + sv * s.E + tv * s.F;
                if (!((z > zz) || (fac < 0))) continue;
                zz = z;
                T n0 = s.nx, n1 = s.ny, n2 = s.nz;
                if (smooth) {
                    double4 q0 = a.vn[s.c0], q1 = a.vn[s.c1], q2 = a.vn[s.c2];
                    T m0 = (T)q0.x + sv * ((T)q1.x - (T)q0.x) + tv * ((T)q2.x - (T)q1.x);
                    T m1 = (T)q0.y + sv * ((T)q1.y - (T)q0.y) + tv * ((T)q2.y - (T)q1.y);
                    T m2 = (T)q0.z + sv * ((T)q1.z - (T)q0.z) + tv * ((T)q2.z - (T)q1.z);
                    T r0 = 0, r1 = 0, r2 = 0;
                    r0 += oa[0] * m0; r0 += oa[1] * m1; r0 += oa[2] * m2;
                    r1 += oa[3] * m0; r1 += oa[4] * m1; r1 += oa[5] * m2;
                    r2 += oa[6] * m0; r2 += oa[7] * m1; r2 += oa[8] * m2;
                    T norm = 0;
                    norm += r0 * r0; norm += r1 * r1; norm += r2 * r2;
                    norm = sqrt(norm);
                    if (norm != (T)0) { r0 /= norm; r1 /= norm; r2 /= norm; }
                    n0 = r0; n1 = r1; n2 = r2;
                }
                if (n2 > (T)0) {
                    cosa = n2;
                    if (bistatic_obs) {
                        cosb = n0 * us0 + n1 * us1 + n2 * us2;
                        if (cosb <= (T)0) cosa = 0;
                    }
                }
                fac = s.f;
            }
        };

        if (count > 0 && count <= a.cap) {
            const int *bin = a.bin_ids + (size_t)(g.tile_base + tile) * a.cap;
            for (int k = tid; k < count; k += RASTER_THREADS) raw[k] = bin[k];
            __syncthreads();
            for (int k = tid; k < count; k += RASTER_THREADS) {
                int v = raw[k], r = 0;
                for (int m = 0; m < count; m++) r += (raw[m] < v);
                ids[r] = v;
            }
            __syncthreads();
            for (int c0 = 0; c0 < count; c0 += STAGE_FACETS) {
                if (tid == 0) s_nst = 0;
                __syncthreads();
                int nst_here = min(STAGE_FACETS, count - c0);
                if (tid < nst_here) {
                    Stage<T> sf;
                    bool ok = stage_facet<T>(a, g, ids[c0 + tid], ti0, ti1, tj0, tj1, sf);
                    if (!ok) { sf.i1 = INT_MAX; sf.i2 = INT_MIN; sf.j1 = INT_MAX; sf.j2 = INT_MIN; sf.f = ids[c0 + tid]; }
                    st[tid] = sf;
                }
                __syncthreads();
                replay(nst_here);
                __syncthreads();
            }
        } else if (count > a.cap) {
            // Bin overflow: stream every facet of the model in index order,
            // keeping those that overlap this tile (order-preserving compaction).
            for (int c0 = 0; c0 < a.nf; c0 += STAGE_FACETS) {
                Stage<T> sf;
                bool ok = false;
                if (tid < STAGE_FACETS && c0 + tid < a.nf)
                    ok = stage_facet<T>(a, g, c0 + tid, ti0, ti1, tj0, tj1, sf);
                unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (lane == 0) s_red[wid][0] = __popc(bal);
                __syncthreads();
                int before = 0, total = 0;
                for (int ww = 0; ww < STAGE_FACETS / 32; ww++) {
                    if (ww < wid) before += s_red[ww][0];
                    total += s_red[ww][0];
                }
                if (ok) st[before + __popc(bal & ((1u << lane) - 1u))] = sf;
                __syncthreads();
                replay(total);
                __syncthreads();
            }
        }

        // ---- outputs of this tile
        const bool covered = inframe && fac >= 0;
        if (inframe && writes_pos) {
            long long p = g.pos_base + (long long)(pi + n) * g.side + (pj + n);
            T *Z = static_cast<T *>(a.pos_z), *CE = static_cast<T *>(a.pos_cose), *CI = static_cast<T *>(a.pos_cosi);
            Z[p] = zz;
            a.pos_f[p] = fac;
            if (g.kind != VIEW_LC_SUN) {
                CE[p] = cosa;
                CI[p] = cosb;
            } else {
                CE[p] = cosa;   // cos(incidence) in the sun view (pos->cosill)
            }
        }
        // covered-pixel bbox (POSrect with (i,i,j,j), posvis.c:278-280)
        int cimin = covered ? pi : INT_MAX, cimax = covered ? pi : INT_MIN;
        int cjmin = covered ? pj : INT_MAX, cjmax = covered ? pj : INT_MIN;
        cimin = warp_min(cimin); cimax = warp_max(cimax);
        cjmin = warp_min(cjmin); cjmax = warp_max(cjmax);
        PixLimits lim = {INT_MAX, INT_MIN, INT_MAX, INT_MIN,
                         SHAPE_HUGENUMBER, -SHAPE_HUGENUMBER, SHAPE_HUGENUMBER, -SHAPE_HUGENUMBER};
        bool lit = false;
        PixDD<T> dd;
        dd.ok = false;
        if (g.kind == VIEW_RADAR && covered) {
            if (a.mark_seen && (double)cosa > a.mincosine_seen)
                a.seen[fac] = 1;
            if (cosa > (T)0) {
                lit = true;
                dd = pixel_dd_setup<T>(g, pi, pj, zz, lim);
            }
        }
        if (g.kind == VIEW_RADAR) {
            // The tile's delay-Doppler footprint is accumulated in shared
            // memory (reusing the bin / stage space, free after the replay)
            // and flushed with one global atomic per touched bin; many pixels
            // of a tile hit the same bins, so this removes most of the
            // contended HBM/L2 atomics.
            int b0 = dd.ok ? dd.idel_min : INT_MAX, b1 = dd.ok ? dd.idel_max : INT_MIN;
            int b2 = dd.ok ? dd.idop_min : INT_MAX, b3 = dd.ok ? dd.idop_max : INT_MIN;
            b0 = warp_min(b0); b1 = warp_max(b1); b2 = warp_min(b2); b3 = warp_max(b3);
            if (lane == 0) { s_box[wid][0] = b0; s_box[wid][1] = b1; s_box[wid][2] = b2; s_box[wid][3] = b3; }
            __syncthreads();
            int r0 = INT_MAX, r1 = INT_MIN, c0 = INT_MAX, c1 = INT_MIN;
            for (int ww = 0; ww < RASTER_THREADS / 32; ww++) {
                r0 = min(r0, s_box[ww][0]); r1 = max(r1, s_box[ww][1]);
                c0 = min(c0, s_box[ww][2]); c1 = max(c1, s_box[ww][3]);
            }
            T *fit = static_cast<T *>(a.fit) + g.fit_base;
            if (r0 != INT_MAX) {
                const int nr = r1 - r0 + 1, nc = c1 - c0 + 1;
                const long long cells = (long long)nr * nc;
                T *box = reinterpret_cast<T *>(smem);
                if (cells <= (long long)(a.smem_bytes / sizeof(T))) {
                    for (long long k = tid; k < cells; k += RASTER_THREADS) box[k] = (T)0;
                    __syncthreads();
                    if (dd.ok) pixel_dd_scatter<T>(a, g, cosa, dd, box, r0, c0, nc);
                    __syncthreads();
                    for (long long k = tid; k < cells; k += RASTER_THREADS) {
                        T v = box[k];
                        if (v != (T)0) {
                            int rr = (int)(k / nc), cc = (int)(k % nc);
                            atomic_add_any<T>(fit + (long long)(r0 + rr - 1) * g.ndop + (c0 + cc - 1), v);
                        }
                    }
                } else if (dd.ok) {
                    pixel_dd_scatter<T>(a, g, cosa, dd, fit, 1, 1, g.ndop);
                }
            }
        }
        if (lane == 0) {
            s_red[wid][0] = cimin; s_red[wid][1] = cimax; s_red[wid][2] = cjmin; s_red[wid][3] = cjmax;
        }
        unsigned anylit = __ballot_sync(0xffffffffu, lit);
        if (g.kind == VIEW_RADAR) {
            lim.idmin = warp_min(lim.idmin); lim.idmax = warp_max(lim.idmax);
            lim.ipmin = warp_min(lim.ipmin); lim.ipmax = warp_max(lim.ipmax);
            lim.dmin = warp_dmin(lim.dmin); lim.dmax = warp_dmax(lim.dmax);
            lim.pmin = warp_dmin(lim.pmin); lim.pmax = warp_dmax(lim.pmax);
            if (lane == 0) {
                s_redl[wid][0] = anylit ? lim.idmin : INT_MAX; s_redl[wid][1] = anylit ? lim.idmax : INT_MIN;
                s_redl[wid][2] = anylit ? lim.ipmin : INT_MAX; s_redl[wid][3] = anylit ? lim.ipmax : INT_MIN;
                s_redd[wid][0] = lim.dmin; s_redd[wid][1] = lim.dmax;
                s_redd[wid][2] = lim.pmin; s_redd[wid][3] = lim.pmax;
            }
        }
        __syncthreads();
        if (tid == 0) {
            FrameState &S = a.states[item.x];
            int v0 = INT_MAX, v1 = INT_MIN, v2 = INT_MAX, v3 = INT_MIN;
            for (int ww = 0; ww < RASTER_THREADS / 32; ww++) {
                v0 = min(v0, s_red[ww][0]); v1 = max(v1, s_red[ww][1]);
                v2 = min(v2, s_red[ww][2]); v3 = max(v3, s_red[ww][3]);
            }
            if (v0 != INT_MAX) {
                atomicMin(&S.cov_i[0], v0); atomicMax(&S.cov_i[1], v1);
                atomicMin(&S.cov_j[0], v2); atomicMax(&S.cov_j[1], v3);
            }
            if (g.kind == VIEW_RADAR) {
                int l0 = INT_MAX, l1 = INT_MIN, l2 = INT_MAX, l3 = INT_MIN;
                double d0 = SHAPE_HUGENUMBER, d1 = -SHAPE_HUGENUMBER, d2 = SHAPE_HUGENUMBER, d3 = -SHAPE_HUGENUMBER;
                for (int ww = 0; ww < RASTER_THREADS / 32; ww++) {
                    l0 = min(l0, s_redl[ww][0]); l1 = max(l1, s_redl[ww][1]);
                    l2 = min(l2, s_redl[ww][2]); l3 = max(l3, s_redl[ww][3]);
                    d0 = fmin(d0, s_redd[ww][0]); d1 = fmax(d1, s_redd[ww][1]);
                    d2 = fmin(d2, s_redd[ww][2]); d3 = fmax(d3, s_redd[ww][3]);
                }
                if (l0 != INT_MAX) {
                    atomicMin(&S.idellim[0], l0); atomicMax(&S.idellim[1], l1);
                    atomicMin(&S.idoplim[0], l2); atomicMax(&S.idoplim[1], l3);
                    atomicMin(&S.dellim[0], dkey(d0)); atomicMax(&S.dellim[1], dkey(d1));
                    atomicMin(&S.doplim[0], dkey(d2)); atomicMax(&S.doplim[1], dkey(d3));
                    S.any_lit = 1;
                }
            }
        }
        __syncthreads();
    }
}

template <typename T>
inline size_t raster_smem_bytes(int cap)
{
    return (((size_t)2 * cap * sizeof(int) + 15) & ~(size_t)15) + (size_t)STAGE_FACETS * sizeof(Stage<T>);
}

// Called once per device before any launch (not inside stream capture).
template <typename T>
inline cudaError_t configure_raster_t()
{
    return cudaFuncSetAttribute(k_raster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

template <typename T>
inline void launch_raster_t(const RasterArgs &a, cudaStream_t s)
{
    if (a.nwork <= 0) return;
    RasterArgs b = a;
    b.smem_bytes = raster_smem_bytes<T>(a.cap);
    k_raster<T><<<a.nwork, RASTER_THREADS, b.smem_bytes, s>>>(b);
}

}  // namespace shape
