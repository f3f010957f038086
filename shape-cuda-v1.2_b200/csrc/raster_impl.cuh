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

#include <algorithm>
#include <climits>
#include <cstddef>

#include "kernels.h"

// Resident CTAs per SM the register allocation must allow (FP32 / FP32
// exact variant / FP64). The rasters are latency-bound: the FP32 kernel at
// 8 CTAs (32 registers, spills to L1) measured faster than 6 (40), 5 (48)
// and 4 (64) on 64 uneven frames (0.188 ms against 0.195 / 0.194 / 0.210);
// its exact variant, with the error bounds live through the replay, is
// fastest at 6 (0.207 ms against 0.264 at 8, 0.214 at 5, 0.225 at 4; 16
// frames of 511x511: 0.295 against 0.311); FP64 at 4 CTAs (64 registers)
// faster than 3 (80).
#ifndef RASTER_MIN_BLOCKS
#define RASTER_MIN_BLOCKS 8
#endif
#ifndef RASTER_MIN_BLOCKS_EXACT
#define RASTER_MIN_BLOCKS_EXACT 6
#endif
#ifndef RASTER_MIN_BLOCKS_F64
#define RASTER_MIN_BLOCKS_F64 4
#endif
// The warp-independent raster (k_raster_w): its shared memory allows 6
// CTAs per SM in FP32 (40 registers) and 3 in FP64.
#ifndef RASTER_W_MIN_BLOCKS
#define RASTER_W_MIN_BLOCKS 6
#endif
#ifndef RASTER_W_MIN_BLOCKS_F64
#define RASTER_W_MIN_BLOCKS_F64 3
#endif
#ifndef RASTER_RARE_NOINLINE
#define RASTER_RARE_NOINLINE 0
#endif
#if RASTER_RARE_NOINLINE
#define RARE_FN __noinline__
#else
#define RARE_FN __forceinline__
#endif

namespace shape {

// Largest facet bitmap (32-bit words) the bin rank uses: models up to 262144
// facets; larger ones rank by comparisons.
constexpr int BITMAP_MAX_WORDS = 8192;
// Bins of at most STAGE_FACETS facets of models up to this many bitmap
// words (65536 facets) are ranked and staged in one pass (k_raster's fused
// path), with the bitmap in its own shared-memory area.
constexpr int FUSED_RANK_MAX_WORDS = 2048;

// Bytes of the ranked bin at the start of a raster CTA's shared memory,
// rounded up so the staging area after it starts on a 32-byte boundary.
__host__ __device__ inline size_t raster_ids_bytes(int cap)
{
    return ((size_t)cap * 8 + 31) & ~(size_t)31;
}

template <typename T> struct Vec4;
template <> struct Vec4<double> { using type = double4; };
template <> struct Vec4<float> { using type = float4; };

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
        v = (T)L.diff_R * ((T)L.diff_C + 1) * (L.diff_linear ? c : tpow<T>(c, 2 * (T)L.diff_C - 1));
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
            v = (T)L.qs_R * ((T)L.qs_C + 1) * (L.qs_linear ? c : tpow<T>(c, 2 * (T)L.qs_C - 1));
        else v = 0;
        break;
    case SHAPE_RADLAW_GAUSSIAN_COSINE:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * (L.diff_linear ? c : tpow<T>(c, 2 * (T)L.diff_C - 1));
        if (c >= (T)L.qs_cos_cutoff) {
            tan2inc = 1 / (c * c) - 1;
            v += (T)L.qs_R * (T)L.qs_C * texp<T>(-(T)L.qs_C * tan2inc) / (c * c * c * c * c);
        }
        break;
    case SHAPE_RADLAW_HAGFORS_COSINE:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * (L.diff_linear ? c : tpow<T>(c, 2 * (T)L.diff_C - 1));
        if (c >= (T)L.qs_cos_cutoff) {
            sin2inc = 1 - c * c;
            arg = c * c * c * c + (T)L.qs_C * sin2inc;
            v += (T)0.5 * (T)L.qs_R * (T)L.qs_C * tpow<T>(arg, (T)-1.5) / c;
        }
        break;
    case SHAPE_RADLAW_COSINE_COSINE:
        v = (T)L.diff_R * ((T)L.diff_C + 1) * (L.diff_linear ? c : tpow<T>(c, 2 * (T)L.diff_C - 1));
        if (c >= (T)L.qs_cos_cutoff)
            v += (T)L.qs_R * ((T)L.qs_C + 1) * (L.qs_linear ? c : tpow<T>(c, 2 * (T)L.qs_C - 1));
        break;
    default:
        break;
    }
    return v;
}

// One staged facet of a tile (shared memory). bb packs the facet's pixel
// bbox clipped to the tile and relative to its corner (4 bits per bound:
// i1, i2, j1, j2); wmask has bit w set when the bbox meets warp w's 4x8
// pixel block.
//
// The terms the per-pixel test reads are packed in three 4-vectors, so a
// visit loads them with three vector loads (every lane of a warp reads the
// same staged facet: broadcasts, no bank conflicts). FP64 form, posvis's
// own terms: p0 = (v00, v01, A, B), p1 = (den, C, D, v02),
// p2 = (E, F, nx, ny). FP32 form, s, t and the depth above the first corner
// as linear functions of the pixel centre's offset (dx, dy) from that
// corner (tile-relative coordinates): s = a1 dx + a2 dy, t = b1 dx + b2 dy,
// zr = c1 dx + c2 dy, with p0 = (v00, v01, a1, a2), p1 = (b1, b2, c1, c2),
// p2 = (v02 lo, v02 hi, nx, ny), v02 = hi + lo to about 2^-48 of itself.
template <typename T>
struct Stage {
    typename Vec4<T>::type p0, p1, p2;
    // one 16-byte group, read with one vector load per visit
    unsigned bb;         // pixel bbox in the tile as byte bounds (pack_bb)
    float es, et, ez;    // FP32 form: error bounds of the FP32 s, t and depth over the tile
    T nz;                // FP64 form: facet normal in view coordinates (p2.z, p2.w, nz), views without smoothing
    // smoothing: FP64 form, the body-frame vertex normals of the three
    // corners; FP32 form, the view-z component of the interpolated normal
    // as r0 + s r1 + t r2 (its sign decides whether cos(e) changes)
    T q[sizeof(T) == 8 ? 9 : 3];
    int wmask, f;
};
static_assert(offsetof(Stage<float>, bb) % 16 == 0 && offsetof(Stage<double>, bb) % 16 == 0,
              "the bbox / error-bound group is read as one 16-byte vector");

// A facet's bbox in its tile (rows ri1..ri2, columns rj1..rj2) packed so one
// byte-wise comparison tests a pixel: pixel (li, lj) packed by pack_px lies
// inside iff every byte of its word is >= the same byte of the bbox word.
__host__ __device__ inline unsigned pack_bb(int ri1, int ri2, int rj1, int rj2)
{
    return (unsigned)ri1 | ((unsigned)rj1 << 8) | ((unsigned)(15 - ri2) << 16) | ((unsigned)(15 - rj2) << 24);
}
__device__ inline unsigned pack_px(int li, int lj)
{
    return (unsigned)li | ((unsigned)lj << 8) | ((unsigned)(15 - li) << 16) | ((unsigned)(15 - lj) << 24);
}

template <typename T>
__device__ inline typename Vec4<T>::type vec4(T x, T y, T z, T w)
{
    typename Vec4<T>::type v;
    v.x = x; v.y = y; v.z = z; v.w = w;
    return v;
}

// Warp w covers tile rows 4*(w>>1) .. +3 and columns 8*(w&1) .. +7.
__device__ inline int warp_mask_of(int ri1, int ri2, int rj1, int rj2)
{
    int m = 0;
#pragma unroll
    for (int w = 0; w < RASTER_THREADS / 32; w++) {
        int r0 = 4 * (w >> 1), c0 = 8 * (w & 1);
        if (ri1 <= r0 + 3 && ri2 >= r0 && rj1 <= c0 + 7 && rj2 >= c0) m |= 1 << w;
    }
    return m;
}

// Facet terms of the s, t, z expressions (src/shape/posvis.c:210-228) and,
// for views without smoothing, the facet normal in view coordinates
// (src/shape/posvis.c:146-148). Both forms stage from the FP64 view-frame
// vertices. The FP32 form stores the corner position relative to the tile
// origin (ox, oy), the edge differences and 1/den rounded from FP64 values,
// so its per-pixel arithmetic works on small, accurately rounded numbers.
template <typename T>
__device__ void stage_fill(const RasterArgs &a, const FrameGeom &g, int f, Stage<T> &s, double ox, double oy)
{
    const double4 *vt = static_cast<const double4 *>(a.vt) + g.vt_base;
    int4 c = a.fvi[f];
    double4 p0 = vt[c.x], p1 = vt[c.y], p2 = vt[c.z];
    T E, F;
    if constexpr (sizeof(T) == 8) {
        const T A = p2.y - p1.y;
        const T B = p2.x - p1.x;
        const T C = p1.x - p0.x;
        const T D = p1.y - p0.y;
        E = p1.z - p0.z;
        F = p2.z - p1.z;
        const T den = (T)1 / (C * A - B * D);
        s.p0 = vec4<T>(p0.x, p0.y, A, B);
        s.p1 = vec4<T>(den, C, D, p0.z);
        (void)ox; (void)oy;
    } else {
        // the linear coefficients in FP64 from posvis's terms, rounded once
        const double A = p2.y - p1.y, B = p2.x - p1.x, C = p1.x - p0.x, D = p1.y - p0.y;
        const double Ez = p1.z - p0.z, Fz = p2.z - p1.z;
        const double den = 1.0 / (C * A - B * D);
        const double V0 = p0.x - ox, V1 = p0.y - oy;
        const double a1 = den * A, a2 = -den * B;
        const double b1 = -den * D, b2 = den * C;
        const double c1 = Ez * a1 + Fz * b1, c2 = Ez * a2 + Fz * b2;
        s.p0 = vec4<T>((T)V0, (T)V1, (T)a1, (T)a2);
        s.p1 = vec4<T>((T)b1, (T)b2, (T)c1, (T)c2);
        // p2 = (v02 lo, v02 hi, nx, ny): the corner depth as a float pair,
        // the rounded value and its rounding error
        F = (T)p0.z;
        E = (T)(p0.z - (double)F);
        // Bounds on the FP32 values' error at any pixel centre of the tile
        // (x, y in [0, 16 kmpp)): 8 units of 2^-24 of the terms' magnitudes
        // (the offsets' rounding, the rounded coefficients, a product and a
        // fused multiply-add; the depth's add); at least 1e-9, so a value
        // past twice its bound also clears posvis's 1e-10 tolerance.
        const double xs = 16.0 * g.kmpp + fabs(V0) + fabs(V1), u = 8.0 / 16777216.0;
        s.es = (float)fmax(1e-9, u * (fabs(a1) + fabs(a2)) * xs);
        s.et = (float)fmax(1e-9, u * (fabs(b1) + fabs(b2)) * xs);
        s.ez = (float)(u * (fabs(p0.z) + (fabs(c1) + fabs(c2)) * xs));
    }
    s.f = f;
    if (g.smooth) {
        double4 q0 = a.vn[c.x], q1 = a.vn[c.y], q2 = a.vn[c.z];
        if constexpr (sizeof(T) == 8) {
            s.q[0] = (T)q0.x; s.q[1] = (T)q0.y; s.q[2] = (T)q0.z;
            s.q[3] = (T)q1.x; s.q[4] = (T)q1.y; s.q[5] = (T)q1.z;
            s.q[6] = (T)q2.x; s.q[7] = (T)q2.y; s.q[8] = (T)q2.z;
        } else {
            // the interpolated normal is linear in (s, t), so is its view-z
            // component: the corners' view-z components in FP64, rounded once
            const double z0 = g.oa[6] * q0.x + g.oa[7] * q0.y + g.oa[8] * q0.z;
            const double z1 = g.oa[6] * q1.x + g.oa[7] * q1.y + g.oa[8] * q1.z;
            const double z2 = g.oa[6] * q2.x + g.oa[7] * q2.y + g.oa[8] * q2.z;
            s.q[0] = (T)z0; s.q[1] = (T)(z1 - z0); s.q[2] = (T)(z2 - z1);
        }
    } else if constexpr (sizeof(T) == 4) {
        // the FP32 form takes the good facet's normal after the replay
        // (good_normal_f32)
        s.p2 = vec4<T>(E, F, (T)0, (T)0);
        s.nz = (T)0;
        return;
    } else {
        double4 nb = a.fn[f];
        double nn[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            nn[r] = 0.0;
            nn[r] += g.oa[3 * r + 0] * nb.x;
            nn[r] += g.oa[3 * r + 1] * nb.y;
            nn[r] += g.oa[3 * r + 2] * nb.z;
        }
        s.p2 = vec4<T>(E, F, (T)nn[0], (T)nn[1]);
        s.nz = (T)nn[2];
        return;
    }
    s.p2 = vec4<T>(E, F, (T)0, (T)0);
}

// Full staging of a facet that did not come from a bin (bin overflow path):
// culling and bounding box as in posvis (src/shape/posvis.c:146-199).
// Returns false when the facet faces away or misses the tile.
template <typename T>
__device__ bool stage_facet(const RasterArgs &a, const FrameGeom &g, int f,
                            int ti0, int ti1, int tj0, int tj1, Stage<T> &s, double ox, double oy)
{
    const double4 *vt = static_cast<const double4 *>(a.vt) + g.vt_base;
    double4 nb = a.fn[f];
    double nz = 0.0;
    nz += g.oa[6] * nb.x;
    nz += g.oa[7] * nb.y;
    nz += g.oa[8] * nb.z;
    if (!(nz > 0.0)) return false;
    int4 c = a.fvi[f];
    double4 p0 = vt[c.x], p1 = vt[c.y], p2 = vt[c.z];
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
    int ri1 = max(i1, ti0) - ti0, ri2 = min(i2, ti1) - ti0;
    int rj1 = max(j1, tj0) - tj0, rj2 = min(j2, tj1) - tj0;
    s.bb = pack_bb(ri1, ri2, rj1, rj2);
    s.wmask = warp_mask_of(ri1, ri2, rj1, rj2);
    stage_fill<T>(a, g, f, s, ox, oy);
    return true;
}

// pos2deldop constants of one frame in the raster's arithmetic type: the
// FP64 raster reads them from FrameGeom, the FP32 raster from the
// host-rounded float copies (FrameGeom::fdd), once per tile.
template <typename T>
struct DDC {
    T delfact, delshift, ax, ay, dopshift, const1, const2, one_over_spb;
    T xincr, yincr, dopdiff_bl, dopdiff_max, dopDC_vig, dopfftlen, kmpp, half_w;
    T spb_over_stride, stride, spb_sq, nsinc2_sq;
};

template <typename T> __device__ inline DDC<T> load_ddc(const FrameGeom &g);
template <> __device__ inline DDC<double> load_ddc<double>(const FrameGeom &g)
{
    DDC<double> c;
    c.delfact = g.delfact; c.delshift = g.delshift; c.ax = g.ax; c.ay = g.ay; c.dopshift = g.dopshift;
    c.const1 = g.const1; c.const2 = g.const2; c.one_over_spb = g.one_over_spb;
    c.xincr = g.xincr; c.yincr = g.yincr; c.dopdiff_bl = g.dopdiff_bl; c.dopdiff_max = g.dopdiff_max;
    c.dopDC_vig = g.dopDC_vig; c.dopfftlen = g.dopfftlen; c.kmpp = g.kmpp; c.half_w = g.sinc2width / 2.0;
    c.spb_over_stride = (double)g.spb_over_stride; c.stride = (double)g.stride;
    c.spb_sq = (double)g.spb_sq; c.nsinc2_sq = (double)g.nsinc2_sq;
    return c;
}
template <> __device__ inline DDC<float> load_ddc<float>(const FrameGeom &g)
{
    const float4 *p = reinterpret_cast<const float4 *>(g.fdd);
    const float4 a = p[0], b = p[1], d = p[2], e = p[3], f = p[4];
    DDC<float> c;
    c.delfact = a.x; c.delshift = a.y; c.ax = a.z; c.ay = a.w;
    c.dopshift = b.x; c.const1 = b.y; c.const2 = b.z; c.one_over_spb = b.w;
    c.xincr = d.x; c.yincr = d.y; c.dopdiff_bl = d.z; c.dopdiff_max = d.w;
    c.dopDC_vig = e.x; c.dopfftlen = e.y; c.kmpp = e.z; c.half_w = e.w;
    c.spb_over_stride = f.x; c.stride = f.y; c.spb_sq = f.z; c.nsinc2_sq = f.w;
    return c;
}

// The view rotation (observer <- body) and the sun direction in the raster's
// arithmetic type: out[0..8] = oa, out[9..11] = usrc.
template <typename T> __device__ inline void load_oa(const FrameGeom &g, T *out);
template <> __device__ inline void load_oa<double>(const FrameGeom &g, double *out)
{
    for (int k = 0; k < 9; k++) out[k] = g.oa[k];
    for (int k = 0; k < 3; k++) out[9 + k] = g.usrc[k];
}
template <> __device__ inline void load_oa<float>(const FrameGeom &g, float *out)
{
    const float4 *p = reinterpret_cast<const float4 *>(g.foa);
    const float4 a = p[0], b = p[1], c = p[2];
    out[0] = a.x; out[1] = a.y; out[2] = a.z; out[3] = a.w;
    out[4] = b.x; out[5] = b.y; out[6] = b.z; out[7] = b.w;
    out[8] = c.x; out[9] = c.y; out[10] = c.z; out[11] = c.w;
}

template <typename T> __device__ inline void atomic_add_fit(T *p, T v);
template <> __device__ inline void atomic_add_fit<double>(double *p, double v) { atomicAdd(p, v); }
template <> __device__ inline void atomic_add_fit<float>(float *p, float v) { atomicAdd(p, v); }

// FP64 delay and Doppler position of a lit pixel; a tile reduces them to the
// frame's limits (dd_bin_limits turns the extremes into bin limits).
struct PixPos {
    double del, dop;
};

// Delay / Doppler position and footprint of one lit POS pixel
// (src/shape/pos2deldop.c:318-367).
template <typename T>
struct PixDD {
    T delPOS, dopPOS, codefactor;
    T ddel0, ddop0, dfrac;     // FP32 form: delPOS - idel_min, dopPOS - idop_min, frac(dopPOS) from FP64
    int ifl;                   // FP32 form: floor(dopPOS) from FP64; column idop's offset is dfrac + (ifl - idop)
    int idel_min, idel_max, idop_min, idop_max;
    bool ok;   // in_bounds: the whole footprint lies inside the frame
};

template <typename T>
__device__ PixDD<T> pixel_dd_setup(const FrameGeom &g, const DDC<T> &k, int x, int y, T z, PixPos &pp)
{
    PixDD<T> d;
    d.delPOS = z * k.delfact + k.delshift;
    const T const1 = k.const1;
    d.idel_min = (int)floor(d.delPOS - const1) + 1;
    d.idel_max = (int)ceil(d.delPOS + const1) - 1;
    d.dopPOS = k.ax * (T)x + k.ay * (T)y + k.dopshift;
    const T dopdiff_max = k.dopdiff_max;
    const T half_w = k.half_w;
    d.idop_min = (int)floor(d.dopPOS - dopdiff_max + 1 - half_w);
    d.idop_max = (int)floor(d.dopPOS + dopdiff_max + half_w);
    // a smeared frame's view adds 1/views of its cross-section (wscale; 1
    // for a frame of one view)
    d.codefactor = ((g.codemethod == SHAPE_CODE_SHORT)
                       ? sinc2<T>((d.dopPOS - k.dopDC_vig) / k.dopfftlen) : (T)1) * (T)g.wscale;
    pp.del = (double)d.delPOS;
    pp.dop = (double)d.dopPOS;
    d.ok = (d.idel_min >= 1) && (d.idel_max <= g.ndel) && (d.idop_min >= 1) && (d.idop_max <= g.ndop) &&
           (d.idel_max - d.idel_min + 1 <= SHAPE_MAXBINS);
    return d;
}

// FP32 form: the pixel's delay and Doppler positions in FP64 from its FP64
// depth (src/shape/pos2deldop.c:318-367), so the bin range and the in-frame
// test are the FP64 form's, and the fractional offsets the FP32 response
// weights take are rounded from FP64 values.
__device__ inline PixDD<float> pixel_dd_setup_x(const FrameGeom &g, int x, int y, double z, PixPos &pp)
{
    PixDD<float> d;
    const double del = z * g.delfact + g.delshift;
    d.idel_min = (int)floor(del - g.const1) + 1;
    d.idel_max = (int)ceil(del + g.const1) - 1;
    const double dop = g.ax * (double)x + g.ay * (double)y + g.dopshift;
    const double half_w = g.sinc2width / 2.0;
    d.idop_min = (int)floor(dop - g.dopdiff_max + 1 - half_w);
    d.idop_max = (int)floor(dop + g.dopdiff_max + half_w);
    d.delPOS = (float)del;
    d.dopPOS = (float)dop;
    d.ddel0 = (float)(del - (double)d.idel_min);
    d.ddop0 = (float)(dop - (double)d.idop_min);
    d.dfrac = (float)(dop - floor(dop));
    d.ifl = (int)floor(dop);
    d.codefactor = ((g.codemethod == SHAPE_CODE_SHORT) ? sinc2<float>((float)((dop - g.dopDC_vig) / g.dopfftlen))
                                                        : 1.0f) * (float)g.wscale;
    pp.del = del;
    pp.dop = dop;
    d.ok = (d.idel_min >= 1) && (d.idel_max <= g.ndel) && (d.idop_min >= 1) && (d.idop_max <= g.ndop) &&
           (d.idel_max - d.idel_min + 1 <= SHAPE_MAXBINS);
    return d;
}

// Bin limits (idel_min, idel_max, idop_min, idop_max) of a set of lit
// pixels from the extremes of their FP64 delay and Doppler positions. Each
// bound is computed per pixel above by the same expression, a non-decreasing
// function of the position (floor/ceil of correctly rounded sums), so its
// extreme over the set is its value at the extreme position: the same
// integers as a min/max over the pixels' own bounds.
__device__ inline void dd_bin_limits(const FrameGeom &g, double dmin, double dmax, double pmin, double pmax, int *l)
{
    const double half_w = g.sinc2width / 2.0;
    l[0] = (int)floor(dmin - g.const1) + 1;
    l[1] = (int)ceil(dmax + g.const1) - 1;
    l[2] = (int)floor(pmin - g.dopdiff_max + 1 - half_w);
    l[3] = (int)floor(pmax + g.dopdiff_max + half_w);
}

template <typename T> __device__ inline void atomic_add_any(T *p, T v) { atomicAdd(p, v); }

// Delay response of image row idel for a pixel at delay bin delPOS
// (src/shape/pos2deldop.c:371-425).
//
// ddel = delPOS - idel. The fast path forms it as (delPOS - idel_min) - r
// with a literal r: both subtractions of integers are exact at these
// magnitudes, so the value is the same as delPOS - (idel_min + r).
template <typename T>
__device__ inline T del_resp(const FrameGeom &g, const DDC<T> &k, T delPOS, T ddel, int idel)
{
    const int spb = g.spb;
    T dc;
    if (g.codemethod != SHAPE_CODE_LONG_ORIG) {
        if (spb == 1) {
            dc = tri2<T>(ddel);
        } else if (spb == 2) {
            T arg = (delPOS - ((T)idel - k.const2)) / k.spb_over_stride;
            dc = tri<T>(arg) + tri<T>(arg - (T)0.5);
            dc *= dc / 4;
        } else {
            dc = 0;
            int m_min = max((int)floor((ddel - k.const2) * k.stride), 0);
            int m_max = min((int)ceil((ddel + k.const1) * k.stride), spb) - 1;
            T arg = (delPOS - ((T)idel - k.const2)) / k.spb_over_stride - (T)m_min * k.one_over_spb;
            for (int m = m_min; m <= m_max; m++) {
                dc += tri<T>(arg);
                arg -= k.one_over_spb;
            }
            dc *= dc / k.spb_sq;
        }
    } else {
        dc = tri2<T>(ddel / k.spb_over_stride);
    }
    return dc;
}

// Mean sinc^2 Doppler response of column idop over nsinc2^2 points
// (src/shape/pos2deldop.c:432-460); s2u = sin^2(pi * frac(dopPOS)) serves
// the nsinc2 == 1 case, where sin^2(pi*(dopPOS - idop)) = s2u.
// ddop = dopPOS - idop, formed like ddel above.
template <typename T>
__device__ inline T dop_resp(const FrameGeom &g, const DDC<T> &k, T dopPOS, T ddop, T s2u, int idop)
{
    const int nsinc2 = g.nsinc2;
    if (nsinc2 == 1) {
        const T t = fabs((T)3.141592653589793 * ddop);
        // FP32 form: the fast quotient (2 ulp; t*t is far from its
        // underflow range) in place of the IEEE division
        if constexpr (sizeof(T) == 4) return (t > 1.0e-4f) ? __fdividef(s2u, t * t) : 1.0f;
        else return (t > 1.0e-4) ? s2u / (t * t) : 1.0;
    }
    if (nsinc2 == 2) {
        T bl = dopPOS + k.dopdiff_bl - (T)idop;
        return (sinc2<T>(bl) + sinc2<T>(bl + k.xincr) + sinc2<T>(bl + k.yincr) +
                sinc2<T>(bl + k.xincr + k.yincr)) / 4;
    }
    T left = dopPOS + k.dopdiff_bl - (T)idop;
    T sm = 0;
    for (int i = 0; i < nsinc2; i++) {
        T arg = left;
        for (int j = 0; j < nsinc2; j++) {
            sm += sinc2<T>(arg);
            arg += k.xincr;
        }
        left += k.yincr;
    }
    return sm / k.nsinc2_sq;
}

// Footprint sizes of the register-resident fast path.
constexpr int FAST_ROWS = 2;
constexpr int FAST_COLS = 8;

// Delay and Doppler response of one pixel and its scatter into `dst`, an
// image whose element (idel, idop) lives at dst[(idel - row0) * stride +
// (idop - col0)] (src/shape/pos2deldop.c:371-496); the raster passes the
// frame's fit image in HBM (row0 = col0 = 1, stride = ndop). Footprints of at
// most FAST_ROWS x FAST_COLS bins (the common LONG_ORIG spb=1 / nsinc2=1 /
// sinc2width<=7 case) keep their weights in registers and scatter through
// fully unrolled, predicated loops, so the lanes of a warp stay converged.
template <typename T, typename A = T>
__device__ void pixel_dd_scatter(const RasterArgs &a, const FrameGeom &g, const DDC<T> &k, T cose,
                                 const PixDD<T> &d, A *dst, int row0, int col0, int stride)
{
    const T delPOS = d.delPOS, dopPOS = d.dopPOS;
    const int idel_min = d.idel_min, idel_max = d.idel_max, idop_min = d.idop_min, idop_max = d.idop_max;
    const int nr = idel_max - idel_min + 1, nc = idop_max - idop_min + 1;
    // FP32 form: the offsets from the FP64 positions (frac + integer)
    constexpr bool f32 = sizeof(T) == 4;
    T s2u = 0;
    if (g.nsinc2 == 1) {
        const T su = tsin<T>((T)3.141592653589793 * (f32 ? d.dfrac : (dopPOS - floor(dopPOS))));
        s2u = su * su;
    }
    auto ddop_of = [&](int idop) -> T { return f32 ? d.dfrac + (T)(d.ifl - idop) : dopPOS - (T)idop; };
    auto ddel_of = [&](int idel) -> T { return f32 ? d.ddel0 - (T)(idel - idel_min) : delPOS - (T)idel; };
    const T kmpp = k.kmpp;
    const T rl = radlaw_dev<T>(a.laws[g.law], cose) * kmpp * kmpp * d.codefactor;
    if (nr <= FAST_ROWS && nc <= FAST_COLS) {
        T dc[FAST_ROWS], pc[FAST_COLS];
        T sdel = 0, sdop = 0;
        const T ddel0 = ddel_of(idel_min), ddop0 = dopPOS - (T)idop_min;
        // the common responses (LONG_ORIG or spb = 1, nsinc2 = 1) written
        // out with del_resp / dop_resp's own operations, so the same values
        if (g.nsinc2 == 1 && (g.codemethod == SHAPE_CODE_LONG_ORIG || g.spb == 1)) {
            const T sos = (g.codemethod == SHAPE_CODE_LONG_ORIG) ? k.spb_over_stride : (T)1;
#pragma unroll
            for (int r = 0; r < FAST_ROWS; r++) {
                dc[r] = (r < nr) ? tri2<T>((ddel0 - (T)r) / sos) : (T)0;
                if (r < nr) sdel += dc[r];
            }
#pragma unroll
            for (int c = 0; c < FAST_COLS; c++) {
                const T t = fabs((T)3.141592653589793 * (f32 ? ddop_of(idop_min + c) : ddop0 - (T)c));
                pc[c] = (c < nc) ? ((t > (T)1.0e-4) ? s2u / (t * t) : (T)1.0) : (T)0;
                if (c < nc) sdop += pc[c];
            }
        } else {
#pragma unroll
            for (int r = 0; r < FAST_ROWS; r++) {
                dc[r] = (r < nr) ? del_resp<T>(g, k, delPOS, ddel0 - (T)r, idel_min + r) : (T)0;
                if (r < nr) sdel += dc[r];
            }
#pragma unroll
            for (int c = 0; c < FAST_COLS; c++) {
                pc[c] = (c < nc) ? dop_resp<T>(g, k, dopPOS, f32 ? ddop_of(idop_min + c) : ddop0 - (T)c, s2u,
                                               idop_min + c) : (T)0;
                if (c < nc) sdop += pc[c];
            }
        }
        // sum of del_c*dop_c over the footprint = (sum del_c) * (sum dop_c)
        // (src/shape/pos2deldop.c:462-466)
        const T amp = rl / (sdel * sdop);
#pragma unroll
        for (int r = 0; r < FAST_ROWS; r++) {
            const T ad = amp * dc[r];
            A *row = dst + (long long)(idel_min + r - row0) * stride + (idop_min - col0);
#pragma unroll
            for (int c = 0; c < FAST_COLS; c++)
                if (r < nr && c < nc) atomic_add_any<A>(row + c, (A)(ad * pc[c]));
        }
        return;
    }
    T del_c[SHAPE_MAXBINS];
    T dop_c[SHAPE_MAXBINS + 1];
    for (int idel = idel_min; idel <= idel_max; idel++)
        del_c[idel - idel_min] = del_resp<T>(g, k, delPOS, ddel_of(idel), idel);
    for (int idop = idop_min; idop <= idop_max; idop++)
        dop_c[min(idop - idop_min, SHAPE_MAXBINS)] = dop_resp<T>(g, k, dopPOS, ddop_of(idop), s2u, idop);
    T sdel = 0, sdop = 0;
    for (int idel = idel_min; idel <= idel_max; idel++) sdel += del_c[idel - idel_min];
    for (int idop = idop_min; idop <= idop_max; idop++) sdop += dop_c[min(idop - idop_min, SHAPE_MAXBINS)];
    const T amp = rl / (sdel * sdop);
    for (int idel = idel_min; idel <= idel_max; idel++) {
        T ad = amp * del_c[idel - idel_min];
        A *row = dst + (long long)(idel - row0) * stride - col0;
        for (int idop = idop_min; idop <= idop_max; idop++)
            atomic_add_any<A>(row + idop, (A)(ad * dop_c[min(idop - idop_min, SHAPE_MAXBINS)]));
    }
}

// The FP32 raster's general scatter (footprints beyond the fast path's, or
// responses other than its two), kept out of line so its arrays and
// constants do not raise the fast path's register use.
// FP32 form, one-row (Doppler) frames: the FP32 weights added in FP64
// (fit64 at the frame's offset): every lit pixel of a spectrum lands in
// the same few hundred bins, so float sums would round thousands of times
// per bin.
static __device__ RARE_FN void pixel_dop_scatter_f32_64(const RasterArgs &a, const FrameGeom &g,
                                                       const DDC<float> &k, float cose, const PixDD<float> &d)
{
    pixel_dd_scatter<float, double>(a, g, k, cose, d, a.fit64 + g.fit_base, 1, 1, g.ndop);
}

static __device__ RARE_FN void pixel_dd_scatter_f32_generic(const RasterArgs &a, const FrameGeom &g,
                                                           const DDC<float> &k, float cose, const PixDD<float> &d,
                                                           float *fit)
{
    pixel_dd_scatter<float>(a, g, k, cose, d, fit, 1, 1, g.ndop);
}

// One footprint row of the FP32 raster straight into the frame's fit image:
// the row's FAST_COLS-wide weights (zero beyond the footprint) are shifted
// by the misalignment m of the first bin (0..3 floats) into the 16-byte
// aligned groups that cover them and land as vector reductions; group lanes
// outside the footprint add zero, which leaves those cells unchanged. The
// shift is two rounds of conditional moves, so the lanes of a warp stay
// converged whatever their misalignments.
__device__ inline void red_row_f32(float4 *base, const float (&w)[FAST_COLS], float ad, int m, int nc)
{
    float v[12];
#pragma unroll
    for (int j = 0; j < 12; j++) v[j] = (j < FAST_COLS) ? w[j] : 0.0f;
    const bool s1 = (m & 1) != 0, s2 = (m & 2) != 0;
#pragma unroll
    for (int j = 11; j >= 0; j--) v[j] = s1 ? (j >= 1 ? v[j - 1] : 0.0f) : v[j];
#pragma unroll
    for (int j = 11; j >= 0; j--) v[j] = s2 ? (j >= 2 ? v[j - 2] : 0.0f) : v[j];
    atomicAdd(base, make_float4(ad * v[0], ad * v[1], ad * v[2], ad * v[3]));
    if (m + nc > 4) atomicAdd(base + 1, make_float4(ad * v[4], ad * v[5], ad * v[6], ad * v[7]));
    if (m + nc > 8) atomicAdd(base + 2, make_float4(ad * v[8], ad * v[9], ad * v[10], ad * v[11]));
}

// FP32 delay-Doppler scatter without a shared-memory accumulator: the same
// weights as pixel_dd_scatter's fast path, added to the fit image in HBM by
// 16-byte vector reductions (at most 2 rows x 3 per pixel instead of 16
// scalar atomics); footprints beyond FAST_ROWS x FAST_COLS and frames with
// other responses take the generic path with scalar atomics.
__device__ inline void pixel_dd_scatter_f32_direct(const RasterArgs &a, const FrameGeom &g, const DDC<float> &k,
                                            float cose, const PixDD<float> &d, float *fit)
{
    const int nr = d.idel_max - d.idel_min + 1, nc = d.idop_max - d.idop_min + 1;
    // the vector path serves the common responses (delay: tri2 of the
    // scaled offset, as LONG_ORIG or spb = 1 give; Doppler: one point per
    // pixel, nsinc2 = 1), written out without the general responses'
    // branches; other frames and larger footprints take the general path
    const bool lean = (g.nsinc2 == 1) && (g.codemethod == SHAPE_CODE_LONG_ORIG || g.spb == 1);
    if (!lean || nr > FAST_ROWS || nc > FAST_COLS) {
        pixel_dd_scatter_f32_generic(a, g, k, cose, d, fit);
        return;
    }
    const float su = sinf(3.141592653589793f * d.dfrac);
    const float s2u = su * su;
    const float rl = radlaw_dev<float>(a.laws[g.law], cose) * k.kmpp * k.kmpp * d.codefactor;
    float dc[FAST_ROWS], pc[FAST_COLS];
    float sdel = 0.0f, sdop = 0.0f;
    const float ddel0 = d.ddel0, ddop0 = d.ddop0;
    // del_resp / dop_resp of these cases (delay offset over spb/stride for
    // LONG_ORIG, over 1 for spb = 1)
    const float sos = (g.codemethod == SHAPE_CODE_LONG_ORIG) ? k.spb_over_stride : 1.0f;
#pragma unroll
    for (int r = 0; r < FAST_ROWS; r++) {
        dc[r] = (r < nr) ? tri2<float>(__fdividef(ddel0 - (float)r, sos)) : 0.0f;
        if (r < nr) sdel += dc[r];
    }
    // the Doppler offset of column c as frac + integer: exact to a float's
    // rounding of its own size, also for the columns next to the pixel
    const int i0 = d.ifl - d.idop_min;
#pragma unroll
    for (int c = 0; c < FAST_COLS; c++) {
        const float t = fabsf(3.141592653589793f * (d.dfrac + (float)(i0 - c)));
        pc[c] = (c < nc) ? ((t > 1.0e-4f) ? __fdividef(s2u, t * t) : 1.0f) : 0.0f;
        if (c < nc) sdop += pc[c];
    }
    (void)ddop0;
    const float amp = __fdividef(rl, sdel * sdop);
#pragma unroll
    for (int r = 0; r < FAST_ROWS; r++) {
        if (r >= nr) break;
        const float ad = amp * dc[r];
        float *cell = fit + (long long)(d.idel_min + r - 1) * g.ndop + (d.idop_min - 1);
        const int mis = (int)((reinterpret_cast<uintptr_t>(cell) >> 2) & 3);
        red_row_f32(reinterpret_cast<float4 *>(cell - mis), pc, ad, mis, nc);
    }
}

// A Doppler pixel whose footprint leaves the spectrum adds its contributions
// to the frame's overflow spectrum instead (src/shape/pos2doppler.c:399-414):
// the same weights as pixel_dd_scatter's generic path (one row, delay
// response 1), bins clipped to the overflow spectrum.
template <typename T>
__device__ RARE_FN void pixel_dop_overflow(const RasterArgs &a, const FrameGeom &g, const DDC<T> &k, T cose,
                                   const PixDD<T> &d)
{
    const int idop_min = d.idop_min, idop_max = d.idop_max;
    T s2u = 0;
    if (g.nsinc2 == 1) {
        T fr;
        if constexpr (sizeof(T) == 4) fr = d.dfrac; else fr = d.dopPOS - floor(d.dopPOS);
        const T su = tsin<T>((T)3.141592653589793 * fr);
        s2u = su * su;
    }
    const T rl = radlaw_dev<T>(a.laws[g.law], cose) * k.kmpp * k.kmpp * d.codefactor;
    T dop_c[SHAPE_MAXBINS + 1];
    for (int idop = idop_min; idop <= idop_max; idop++) {
        T ddop;
        if constexpr (sizeof(T) == 4) ddop = d.dfrac + (T)(d.ifl - idop); else ddop = d.dopPOS - (T)idop;
        dop_c[min(idop - idop_min, SHAPE_MAXBINS)] = dop_resp<T>(g, k, d.dopPOS, ddop, s2u, idop);
    }
    T sdop = 0;
    for (int idop = idop_min; idop <= idop_max; idop++) sdop += dop_c[min(idop - idop_min, SHAPE_MAXBINS)];
    const T amp = rl / ((T)1 * sdop);
    double *ov = a.ovf + g.ovf_base;
    const int idop1 = max(idop_min, -g.idop0), idop2 = min(idop_max, -g.idop0 + DOP_MAXOVERFLOW - 1);
    for (int idop = idop1; idop <= idop2; idop++)
        atomicAdd(ov + idop + g.idop0, (double)(amp * (T)1 * dop_c[min(idop - idop_min, SHAPE_MAXBINS)]));
}

// FP32 form: the FP64 depth of facet c at the pixel centre (x0, y0), with
// the FP64 form's terms and operation order (stage_fill and the visit's s,
// t, z), rounded op by op so no multiply-add is fused: the same value the
// FP64 raster stores for this facet. posmask compares such depths with the
// sun view's, where a few 1e-8 km decide a pixel's shadow.
__device__ inline double facet_depth64(const double4 *vt, int4 c, double x0, double y0)
{
    const double4 p0 = vt[c.x], p1 = vt[c.y], p2 = vt[c.z];
    const double A = __dsub_rn(p2.y, p1.y), B = __dsub_rn(p2.x, p1.x);
    const double C = __dsub_rn(p1.x, p0.x), D = __dsub_rn(p1.y, p0.y);
    const double E = __dsub_rn(p1.z, p0.z), F = __dsub_rn(p2.z, p1.z);
    const double den = 1.0 / __dsub_rn(__dmul_rn(C, A), __dmul_rn(B, D));
    const double dx = __dsub_rn(x0, p0.x), dy = __dsub_rn(y0, p0.y);
    const double sv = __dmul_rn(__dsub_rn(__dmul_rn(dx, A), __dmul_rn(B, dy)), den);
    const double tv = __dmul_rn(__dsub_rn(__dmul_rn(C, dy), __dmul_rn(dx, D)), den);
    return __dadd_rn(__dadd_rn(p0.z, __dmul_rn(sv, E)), __dmul_rn(tv, F));
}

// FP32 form, lightcurve views: cos(e) and cos(i) of a pixel from its good
// facet gf (the last winner whose smoothed normal faced the viewer; the
// winner itself without smoothing) with the FP64 form's values and
// operations, rounded op by op: the interpolated vertex normal at the pixel
// centre, its view coordinates, normalization and the sun direction
// (src/shape/posvis.c:250-274). The brightness sums then equal the FP64
// form's: a lightcurve's chi-square is a small difference of large sums
// (floating calibration, 1 % noise), which magnifies FP32 cosines' rounding.
static __device__ void lc_cos64(const RasterArgs &a, const FrameGeom &g, int gf, double x0, double y0,
                                bool smooth, bool bistatic_obs, double *ce, double *ci)
{
    double n0, n1, n2;
    if (smooth) {
        const double4 *vt = static_cast<const double4 *>(a.vt) + g.vt_base;
        const int4 c = a.fvi[gf];
        const double4 p0 = vt[c.x], p1 = vt[c.y], p2 = vt[c.z];
        const double A = __dsub_rn(p2.y, p1.y), B = __dsub_rn(p2.x, p1.x);
        const double C = __dsub_rn(p1.x, p0.x), D = __dsub_rn(p1.y, p0.y);
        const double den = 1.0 / __dsub_rn(__dmul_rn(C, A), __dmul_rn(B, D));
        const double dx = __dsub_rn(x0, p0.x), dy = __dsub_rn(y0, p0.y);
        const double sv = __dmul_rn(__dsub_rn(__dmul_rn(dx, A), __dmul_rn(B, dy)), den);
        const double tv = __dmul_rn(__dsub_rn(__dmul_rn(C, dy), __dmul_rn(dx, D)), den);
        const double4 q0 = a.vn[c.x], q1 = a.vn[c.y], q2 = a.vn[c.z];
        const double m0 = __dadd_rn(__dadd_rn(q0.x, __dmul_rn(sv, __dsub_rn(q1.x, q0.x))),
                                    __dmul_rn(tv, __dsub_rn(q2.x, q1.x)));
        const double m1 = __dadd_rn(__dadd_rn(q0.y, __dmul_rn(sv, __dsub_rn(q1.y, q0.y))),
                                    __dmul_rn(tv, __dsub_rn(q2.y, q1.y)));
        const double m2 = __dadd_rn(__dadd_rn(q0.z, __dmul_rn(sv, __dsub_rn(q1.z, q0.z))),
                                    __dmul_rn(tv, __dsub_rn(q2.z, q1.z)));
        double r[3];
        for (int k = 0; k < 3; k++)
            r[k] = __dadd_rn(__dadd_rn(__dmul_rn(g.oa[3 * k], m0), __dmul_rn(g.oa[3 * k + 1], m1)),
                             __dmul_rn(g.oa[3 * k + 2], m2));
        const double norm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(r[0], r[0]), __dmul_rn(r[1], r[1])),
                                                 __dmul_rn(r[2], r[2])));
        if (norm != 0.0)
            for (int k = 0; k < 3; k++) r[k] = __ddiv_rn(r[k], norm);
        n0 = r[0]; n1 = r[1]; n2 = r[2];
    } else {
        const double4 nb = a.fn[gf];
        double nn[3];
        for (int k = 0; k < 3; k++)
            nn[k] = __dadd_rn(__dadd_rn(__dmul_rn(g.oa[3 * k], nb.x), __dmul_rn(g.oa[3 * k + 1], nb.y)),
                              __dmul_rn(g.oa[3 * k + 2], nb.z));
        n0 = nn[0]; n1 = nn[1]; n2 = nn[2];
    }
    *ce = 0.0;
    *ci = 0.0;
    if (n2 > 0.0) {
        *ce = n2;
        if (bistatic_obs) {
            *ci = __dadd_rn(__dadd_rn(__dmul_rn(n0, g.usrc[0]), __dmul_rn(n1, g.usrc[1])), __dmul_rn(n2, g.usrc[2]));
            if (*ci <= 0.0) *ce = 0.0;
        }
    }
}

// FP32 form: the normal of a pixel's good facet gf at its barycentric
// coordinates (sv, tv) of that visit: the interpolated body-frame vertex
// normal with the raster's rounded corner normals (smoothing), or the facet
// normal in view coordinates as staging rounds it. The replay keeps only
// (gf, sv, tv) per pixel, so a visit costs two multiply-adds for the sign.
__device__ inline void good_normal_f32(const RasterArgs &a, const FrameGeom &g, int gf, float sv, float tv,
                                       bool smooth, float &m0, float &m1, float &m2)
{
    if (smooth) {
        const int4 c = a.fvi[gf];
        const double4 q0 = a.vn[c.x], q1 = a.vn[c.y], q2 = a.vn[c.z];
        const float ax = (float)q0.x, ay = (float)q0.y, az = (float)q0.z;
        const float bx = (float)q1.x, by = (float)q1.y, bz = (float)q1.z;
        const float cx = (float)q2.x, cy = (float)q2.y, cz = (float)q2.z;
        m0 = ax + sv * (bx - ax) + tv * (cx - bx);
        m1 = ay + sv * (by - ay) + tv * (cy - by);
        m2 = az + sv * (bz - az) + tv * (cz - bz);
    } else {
        const double4 nb = a.fn[gf];
        double nn[3];
#pragma unroll
        for (int r = 0; r < 3; r++) {
            nn[r] = 0.0;
            nn[r] += g.oa[3 * r + 0] * nb.x;
            nn[r] += g.oa[3 * r + 1] * nb.y;
            nn[r] += g.oa[3 * r + 2] * nb.z;
        }
        m0 = (float)nn[0]; m1 = (float)nn[1]; m2 = (float)nn[2];
    }
}

// FP32 form, rare path: posvis at one pixel by the FP64 form's rules (the
// FP64 visit's s, t, depth and tolerance, rounded op by op; its update rule
// and order-dependent smoothed normal), over the tile's bin in facet order.
// ids: the bin's (facet, packed tile bbox) entries, sorted; (li, lj): the
// pixel in the tile; (x0, y0): its centre. Returns the winner's facet
// (-1: none) and writes its FP64 depth and the cos(e) state.
static __device__ RARE_FN int pixel_posvis64(const RasterArgs &a, const FrameGeom &g, const int2 *ids,
                                                  int count, int li, int lj, double x0, double y0, double *zz,
                                                  bool *good, float *gm, int *gf)
{
    const double4 *vt = static_cast<const double4 *>(a.vt) + g.vt_base;
    double zw = -SHAPE_HUGENUMBER;
    int fac = -1;
    for (int k = 0; k < count; k++) {
        const int2 e = ids[k];
        const int b = e.y;
        if (li < (b & 15) || li > ((b >> 4) & 15) || lj < ((b >> 8) & 15) || lj > ((b >> 12) & 15)) continue;
        const int4 c = a.fvi[e.x];
        const double4 p0 = vt[c.x], p1 = vt[c.y], p2 = vt[c.z];
        const double A = __dsub_rn(p2.y, p1.y), B = __dsub_rn(p2.x, p1.x);
        const double C = __dsub_rn(p1.x, p0.x), D = __dsub_rn(p1.y, p0.y);
        const double E = __dsub_rn(p1.z, p0.z), F = __dsub_rn(p2.z, p1.z);
        const double den = 1.0 / __dsub_rn(__dmul_rn(C, A), __dmul_rn(B, D));
        const double dx = __dsub_rn(x0, p0.x), dy = __dsub_rn(y0, p0.y);
        const double sv = __dmul_rn(__dsub_rn(__dmul_rn(dx, A), __dmul_rn(B, dy)), den);
        if (!((sv >= -SHAPE_SMALLVAL) && (sv <= __dadd_rn(1.0, SHAPE_SMALLVAL)))) continue;
        const double tv = __dmul_rn(__dsub_rn(__dmul_rn(C, dy), __dmul_rn(dx, D)), den);
        if (!((tv >= -SHAPE_SMALLVAL) && (tv <= __dadd_rn(sv, SHAPE_SMALLVAL)))) continue;
        const double z = __dadd_rn(__dadd_rn(p0.z, __dmul_rn(sv, E)), __dmul_rn(tv, F));
        if (!((z > zw) || (fac < 0))) continue;
        zw = z;
        fac = e.x;
        if (g.smooth) {
            const double4 q0 = a.vn[c.x], q1 = a.vn[c.y], q2 = a.vn[c.z];
            const double m0 = __dadd_rn(__dadd_rn(q0.x, __dmul_rn(sv, __dsub_rn(q1.x, q0.x))),
                                        __dmul_rn(tv, __dsub_rn(q2.x, q1.x)));
            const double m1 = __dadd_rn(__dadd_rn(q0.y, __dmul_rn(sv, __dsub_rn(q1.y, q0.y))),
                                        __dmul_rn(tv, __dsub_rn(q2.y, q1.y)));
            const double m2 = __dadd_rn(__dadd_rn(q0.z, __dmul_rn(sv, __dsub_rn(q1.z, q0.z))),
                                        __dmul_rn(tv, __dsub_rn(q2.z, q1.z)));
            double r2 = 0.0;
            r2 = __dadd_rn(r2, __dmul_rn(g.oa[6], m0));
            r2 = __dadd_rn(r2, __dmul_rn(g.oa[7], m1));
            r2 = __dadd_rn(r2, __dmul_rn(g.oa[8], m2));
            if (r2 > 0.0) { *good = true; gm[0] = (float)m0; gm[1] = (float)m1; gm[2] = (float)m2; *gf = e.x; }
        } else {
            const double4 nb = a.fn[e.x];
            double nn[3];
            for (int r = 0; r < 3; r++) {
                nn[r] = 0.0;
                nn[r] = __dadd_rn(nn[r], __dmul_rn(g.oa[3 * r + 0], nb.x));
                nn[r] = __dadd_rn(nn[r], __dmul_rn(g.oa[3 * r + 1], nb.y));
                nn[r] = __dadd_rn(nn[r], __dmul_rn(g.oa[3 * r + 2], nb.z));
            }
            *good = true; gm[0] = (float)nn[0]; gm[1] = (float)nn[1]; gm[2] = (float)nn[2]; *gf = e.x;
        }
    }
    *zz = zw;
    return fac;
}

// Warp-wide extremes with the hardware warp reduction (one instruction per
// 32-bit word); 64-bit order-preserving keys (dkey) reduce their high words
// first, then the low words of the lanes holding the extreme high word.
__device__ inline int warp_min(int v) { return __reduce_min_sync(0xffffffffu, v); }
__device__ inline int warp_max(int v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ inline unsigned long long warp_kmin(unsigned long long k)
{
    const unsigned hi = __reduce_min_sync(0xffffffffu, (unsigned)(k >> 32));
    const unsigned lo = __reduce_min_sync(0xffffffffu, ((unsigned)(k >> 32) == hi) ? (unsigned)k : 0xffffffffu);
    return ((unsigned long long)hi << 32) | lo;
}
__device__ inline unsigned long long warp_kmax(unsigned long long k)
{
    const unsigned hi = __reduce_max_sync(0xffffffffu, (unsigned)(k >> 32));
    const unsigned lo = __reduce_max_sync(0xffffffffu, ((unsigned)(k >> 32) == hi) ? (unsigned)k : 0u);
    return ((unsigned long long)hi << 32) | lo;
}

// Bytes of the staging area after the ranked bin (32-byte multiple): the
// staged facets, or while a bin is ranked the unfused path's bitmap, prefix
// counts and raw bin. The fused path's bitmap follows it.
template <typename T>
__host__ __device__ inline size_t raster_stage_bytes(int cap, int nf)
{
    const size_t nw = ((size_t)nf + 31) / 32;
    const size_t scratch = (nw <= (size_t)BITMAP_MAX_WORDS ? 8 * nw : 0) + (size_t)cap * sizeof(int2);
    const size_t st = (size_t)STAGE_FACETS * sizeof(Stage<T>);
    return ((st > scratch ? st : scratch) + 31) & ~(size_t)31;
}

// The tile raster. EXACT (FP32 form, lightcurve views): a pixel with a
// decision within FP32 error is redone by the FP64 form's rules, so facet
// assignment, depth and the shadow test's inputs are the FP64 form's;
// without it (radar views) the FP32 test is posvis's with FP32 values.
template <typename T, bool EXACT, bool LCV = false>
__global__ void __launch_bounds__(RASTER_THREADS, sizeof(T) == 8 ? RASTER_MIN_BLOCKS_F64
                                                  : (EXACT ? RASTER_MIN_BLOCKS_EXACT : RASTER_MIN_BLOCKS))
k_raster(RasterArgs a)
{
    grid_dep_wait();
    extern __shared__ __align__(32) unsigned char smem[];
    // dynamic shared memory: the ranked bin, then the staging area, which
    // holds the facet bitmap, its prefix counts and the raw bin while the bin
    // is ranked (raster_smem_bytes sizes it for both uses)
    int2 *ids = reinterpret_cast<int2 *>(smem);
    Stage<T> *st = reinterpret_cast<Stage<T> *>(smem + raster_ids_bytes(a.cap));
    __shared__ int s_red[RASTER_THREADS / 32][4];
    __shared__ unsigned long long s_redk[RASTER_THREADS / 32][4];
    __shared__ int s_scan[RASTER_THREADS / 32];
    __shared__ unsigned char s_perm[STAGE_FACETS];
    __shared__ double s_pz[TILE_PIX];
    __shared__ T s_pc[TILE_PIX];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    // warp wid owns a 4x8 block of the 16x16 tile
    const int li = 4 * (wid >> 1) + (lane >> 3), lj = 8 * (wid & 1) + (lane & 7);

    for (int w = blockIdx.x; w < a.nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const FrameGeom &g = a.geoms[item.x];
        const int tile = item.y;
        const int tx = tile / g.tiles_x, ty = tile % g.tiles_x;
        const int n = g.n;
        const int ti0 = -n + tx * TILE_W, tj0 = -n + ty * TILE_W;
        const int ti1 = min(ti0 + TILE_W - 1, n), tj1 = min(tj0 + TILE_W - 1, n);
        const int pi = ti0 + li, pj = tj0 + lj;
        const bool inframe = (pi <= n) && (pj <= n);
        const int count = a.bin_count[g.tile_base + tile];
        const bool writes_pos = (g.kind != VIEW_RADAR) || a.keep_pos;
        if (count == 0 && !writes_pos) continue;

        // pixel centre: absolute (FP64 form) or relative to the tile origin
        // (FP32 form, matching the tile-relative staged corners)
        const double ox = (double)ti0 * g.kmpp, oy = (double)tj0 * g.kmpp;
        const T x0 = (sizeof(T) == 8) ? (T)pi * (T)g.kmpp : (T)((double)li * g.kmpp);
        const T x1 = (sizeof(T) == 8) ? (T)pj * (T)g.kmpp : (T)((double)lj * g.kmpp);
        T zz = (T)(-SHAPE_HUGENUMBER), cosa = 0, cosb = 0;
        int fac = -1;
        if constexpr (sizeof(T) == 8) {
            // a single view accumulating over earlier calls (posvis over
            // model components): the pixel starts from what the images hold
            if (a.accumulate && inframe) {
                const long long p = g.pos_base + (long long)(pi + n) * g.side + (pj + n);
                zz = static_cast<const double *>(a.pos_z)[p];
                fac = a.pos_f[p];
                cosa = static_cast<const T *>(a.pos_cose)[p];
                if (g.kind != VIEW_LC_SUN) cosb = static_cast<const T *>(a.pos_cosi)[p];
            }
        }
        T zze = 0;       // FP32 form: the winner's depth error bound
        T zlo = 0;       // FP32 form: the winner's depth is zz + zlo (two floats)
        bool amb = false;   // FP32 form: a decision within FP32 error (pixel_posvis64 redoes it)
        bool good = false;
        T gm0 = 0, gm1 = 0, gm2 = 0;
        int gfac = -1;             // FP32 form: the good facet and its (s, t) at this pixel
        float gsv = 0.0f, gtv = 0.0f;
        bool gready = false;       // FP32 form: gm0..2 already set (the FP64 redo)
        const bool smooth = g.smooth != 0;
        const bool bistatic_obs = (g.kind == VIEW_LC_OBS);
        // FP32 form, lightcurve views (their own launch, LCV): the good
        // facet's index rides in gm0's bits, and the cosines are recomputed
        // from it in FP64 (lc_cos64); radar launches compile this out
        const bool lcv = (sizeof(T) == 4) && EXACT && LCV && (g.kind != VIEW_RADAR);
        const T oa6 = (T)g.oa[6], oa7 = (T)g.oa[7], oa8 = (T)g.oa[8];

        // Apply posvis's update rule for one staged facet at this pixel.
        const unsigned pxw = pack_px(li, lj);
        auto visit = [&](const Stage<T> &s) {
            T sv, tv, z, zr = 0;
            if constexpr (sizeof(T) == 8) {
                if (__vcmpgeu4(pxw, s.bb) != 0xffffffffu) return;   // pixel outside the facet's bbox
                const auto p0 = s.p0, p1 = s.p1;
                const T dx = x0 - p0.x, dy = x1 - p0.y;
                sv = (dx * p0.z - p0.w * dy) * p1.x;
                if (!((sv >= (T)-SHAPE_SMALLVAL) && (sv <= (T)1.0 + (T)SHAPE_SMALLVAL))) return;
                tv = (p1.y * dy - dx * p1.z) * p1.x;
                if (!((tv >= (T)-SHAPE_SMALLVAL) && (tv <= sv + (T)SHAPE_SMALLVAL))) return;
                const auto p2 = s.p2;
                z = p1.w + sv * p2.x + tv * p2.y;
                if (!((z > zz) || (fac < 0))) return;
            } else {
                // FP32 test without early exits (a warp runs every step for
                // some lane anyway). A value within its error bound of a
                // boundary of the test, or a depth within the bounds of the
                // winner's, marks the pixel ambiguous: after the replay it is
                // redone by the FP64 form's own rules (pixel_posvis64), so the
                // FP32 form assigns facets as the FP64 form does.
                const auto p0 = s.p0, p1 = s.p1, p2 = s.p2;
                const float4 be = *reinterpret_cast<const float4 *>(&s.bb);   // bb, es, et, ez
                const bool inb = __vcmpgeu4(pxw, __float_as_uint(be.x)) == 0xffffffffu;   // pixel in the facet's bbox
                const T dx = x0 - p0.x, dy = x1 - p0.y;
                sv = fmaf(p0.z, dx, p0.w * dy);
                tv = fmaf(p1.x, dx, p1.y * dy);
                zr = fmaf(p1.z, dx, p1.w * dy);
                z = p2.y + zr;
                const T es = be.y, et = be.z, est = es + et;
                if constexpr (EXACT) {
                    const bool out = !inb || (sv < -2 * es) || (sv > 1 + 2 * es) || (tv < -2 * et) ||
                                     (tv > sv + 2 * est);
                    if (out) return;
                    const bool sure = (sv >= es) && (sv <= 1 - es) && (tv >= et) && (tv <= sv - est);
                    const bool near = (fac >= 0) && (fabsf(z - zz) <= be.w + zze);
                    amb = amb || !sure || near;
                    if (!((z > zz) || (fac < 0))) return;
                    zze = be.w;
                } else {
                    // posvis's own tolerance: a wider one (the error bounds)
                    // also covers pixels just outside the silhouette, which
                    // measured worse than the rare pixel on a shared edge
                    // that both facets' FP32 tests miss
                    const bool in = inb && (sv >= (T)-SHAPE_SMALLVAL) && (sv <= (T)1.0 + (T)SHAPE_SMALLVAL) &&
                                    (tv >= (T)-SHAPE_SMALLVAL) && (tv <= sv + (T)SHAPE_SMALLVAL);
                    if (!(in && ((z > zz) || (fac < 0)))) return;
                }
            }
            const auto p2 = s.p2;
            zz = z;
            fac = s.f;
            if constexpr (sizeof(T) == 4) {
                // the depth as a float pair: the rounding error of v02 hi + zr
                // (two-sum) plus v02's low part, so radar views get their
                // depth to a few 1e-9 km without an FP64 recomputation
                const float bv = z - p2.y;
                zlo = ((p2.y - (z - bv)) + (zr - bv)) + p2.x;
            }
            // cos(e) changes only when the smoothed normal faces the viewer
            // (posvis.c:265). Its sign is that of the view-z component before
            // normalization, so a win records the body-frame interpolated
            // normal and the last qualifying one is normalized once, below.
            if constexpr (sizeof(T) == 4) {
                // FP32: the sign of the normal's view-z component from the
                // staged linear form (the coefficients' rounding, the s and t
                // errors times coefficients below 2, and two multiply-adds
                // stay inside the bound); the normal itself is formed once,
                // after the replay, from (facet, s, t)
                if (smooth) {
                    const T r2 = s.q[0] + sv * s.q[1] + tv * s.q[2];
                    if constexpr (EXACT) amb = amb || (fabsf(r2) <= 4 * (s.es + s.et) + 3e-6f);
                    if (r2 > (T)0) { good = true; gfac = s.f; gsv = sv; gtv = tv; }
                } else {
                    good = true; gfac = s.f;
                }
            } else if (smooth) {
                const T m0 = s.q[0] + sv * (s.q[3] - s.q[0]) + tv * (s.q[6] - s.q[3]);
                const T m1 = s.q[1] + sv * (s.q[4] - s.q[1]) + tv * (s.q[7] - s.q[4]);
                const T m2 = s.q[2] + sv * (s.q[5] - s.q[2]) + tv * (s.q[8] - s.q[5]);
                T r2 = 0;
                r2 += oa6 * m0; r2 += oa7 * m1; r2 += oa8 * m2;
                if (r2 > (T)0) { good = true; gm0 = m0; gm1 = m1; gm2 = m2; }
            } else {
                good = true; gm0 = p2.z; gm1 = p2.w; gm2 = s.nz;
            }
        };
        // Each warp walks only the staged facets whose bbox meets its block,
        // in staging (= facet index) order.
        // order: the staged slots in facet-index order (fused path), or
        // null when the slots are already in that order
        auto replay = [&](int nst, const unsigned char *order) {
            for (int base = 0; base < nst; base += 32) {
                const int k = base + lane;
                const int slot = (k < nst) ? (order ? (int)order[k] : k) : 0;
                const bool hit = (k < nst) && ((st[slot].wmask >> wid) & 1);
                unsigned m = __ballot_sync(0xffffffffu, hit);
                while (m) {
                    const int b = __ffs(m) - 1;
                    m &= m - 1;
                    visit(st[__shfl_sync(0xffffffffu, slot, b)]);
                }
            }
        };

        if (count > 0 && count <= a.cap) {
            const int2 *bin = a.bin_ids + (size_t)(g.tile_base + tile) * a.cap;
            const int nw = (a.nf + 31) >> 5;
            if (count <= STAGE_FACETS && nw <= FUSED_RANK_MAX_WORDS) {
            // Fused rank and staging (a bin that fits one staging pass): each
            // of the first `count` threads loads one bin entry, marks its
            // facet in a bitmap of the bin's facets and stages the facet in
            // its own slot, so the staging loads overlap the marking; the
            // bitmap's prefix counts then give each facet its rank (the
            // number of the bin's facets below it), and the replay walks the
            // slots in rank order, which is facet-index order.
            unsigned *W = reinterpret_cast<unsigned *>(smem + raster_ids_bytes(a.cap) +
                                                       raster_stage_bytes<T>(a.cap, a.nf));
            int *P = reinterpret_cast<int *>(W + nw);
            for (int w = tid; w < nw; w += RASTER_THREADS) W[w] = 0u;
            __syncthreads();
            int2 e = make_int2(0, 0);
            if (tid < count) {
                e = bin[tid];
                atomicOr(&W[e.x >> 5], 1u << (e.x & 31));
                Stage<T> sf;
                const int bb = e.y;
                sf.bb = pack_bb(bb & 15, (bb >> 4) & 15, (bb >> 8) & 15, (bb >> 12) & 15);
                sf.wmask = warp_mask_of(bb & 15, (bb >> 4) & 15, (bb >> 8) & 15, (bb >> 12) & 15);
                stage_fill<T>(a, g, e.x, sf, ox, oy);
                st[tid] = sf;
            }
            __syncthreads();
            // P[w]: the set bits of the words before w within the owning
            // warp's words (each thread owns a run of wpt words); s_scan:
            // the warps' totals
            const int wpt = (nw + RASTER_THREADS - 1) / RASTER_THREADS;
            const int w0 = min(tid * wpt, nw), w1 = min(w0 + wpt, nw);
            int run = 0;
            for (int w = w0; w < w1; w++) run += __popc(W[w]);
            int inc = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            if (lane == 31) s_scan[wid] = inc;
            int before = inc - run;
            for (int w = w0; w < w1; w++) {
                P[w] = before;
                before += __popc(W[w]);
            }
            __syncthreads();
            if (tid < count) {
                const int w = e.x >> 5;
                const int owner = (w / wpt) >> 5;
                int r = P[w] + __popc(W[w] & ((1u << (e.x & 31)) - 1u));
                for (int ww = 0; ww < owner; ww++) r += s_scan[ww];
                ids[r] = e;
                s_perm[r] = (unsigned char)tid;
            }
            __syncthreads();
            replay(count, s_perm);
            } else {
            // The bin in facet-index order (posvis walks facets in index
            // order). A bin's facets are distinct, so a facet's rank is the
            // number of set bits below it in a bitmap of the bin's facets:
            // O(nf/32 + count) per tile. The bitmap, its per-word prefix
            // counts and the raw bin live in the staging area, idle until
            // staging starts; models too large for a bitmap rank by
            // comparisons.
            if (nw <= BITMAP_MAX_WORDS) {
                unsigned *W = reinterpret_cast<unsigned *>(st);
                int *P = reinterpret_cast<int *>(W + nw);
                int2 *raw = reinterpret_cast<int2 *>(P + nw);
                for (int w = tid; w < nw; w += RASTER_THREADS) W[w] = 0u;
                __syncthreads();
                for (int k = tid; k < count; k += RASTER_THREADS) {
                    const int2 v = bin[k];
                    raw[k] = v;
                    atomicOr(&W[v.x >> 5], 1u << (v.x & 31));
                }
                __syncthreads();
                // exclusive prefix of the words' popcounts: a contiguous run
                // of words per thread, then a block scan of the run totals
                const int wpt = (nw + RASTER_THREADS - 1) / RASTER_THREADS;
                const int w0 = min(tid * wpt, nw), w1 = min(w0 + wpt, nw);
                int run = 0;
                for (int w = w0; w < w1; w++) run += __popc(W[w]);
                int inc = run;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += t;
                }
                if (lane == 31) s_scan[wid] = inc;
                __syncthreads();
                int before = inc - run;
                for (int ww = 0; ww < wid; ww++) before += s_scan[ww];
                for (int w = w0; w < w1; w++) {
                    P[w] = before;
                    before += __popc(W[w]);
                }
                __syncthreads();
                for (int k = tid; k < count; k += RASTER_THREADS) {
                    const int2 v = raw[k];
                    const int w = v.x >> 5;
                    ids[P[w] + __popc(W[w] & ((1u << (v.x & 31)) - 1u))] = v;
                }
            } else {
                int2 *raw = reinterpret_cast<int2 *>(st);
                for (int k = tid; k < count; k += RASTER_THREADS) raw[k] = bin[k];
                __syncthreads();
                for (int k = tid; k < count; k += RASTER_THREADS) {
                    int2 v = raw[k];
                    int r = 0;
                    for (int m = 0; m < count; m++) r += (raw[m].x < v.x);
                    ids[r] = v;
                }
            }
            __syncthreads();
            for (int c0 = 0; c0 < count; c0 += STAGE_FACETS) {
                const int nst = min(STAGE_FACETS, count - c0);
                if (tid < nst) {
                    const int2 e = ids[c0 + tid];
                    Stage<T> sf;
                    const int bb = e.y;
                    sf.bb = pack_bb(bb & 15, (bb >> 4) & 15, (bb >> 8) & 15, (bb >> 12) & 15);
                    sf.wmask = warp_mask_of(bb & 15, (bb >> 4) & 15, (bb >> 8) & 15, (bb >> 12) & 15);
                    stage_fill<T>(a, g, e.x, sf, ox, oy);
                    st[tid] = sf;
                }
                __syncthreads();
                replay(nst, nullptr);
                __syncthreads();
            }
            }
        } else if (count > a.cap) {
            // Bin overflow: stream every facet of the model in index order,
            // keeping those that overlap this tile (order-preserving compaction).
            for (int c0 = 0; c0 < a.nf; c0 += STAGE_FACETS) {
                Stage<T> sf;
                bool ok = false;
                if (tid < STAGE_FACETS && c0 + tid < a.nf)
                    ok = stage_facet<T>(a, g, c0 + tid, ti0, ti1, tj0, tj1, sf, ox, oy);
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
                replay(total, nullptr);
                __syncthreads();
            }
        }

        // FP32 form: a pixel with a decision within FP32 error is redone by
        // the FP64 form's rules over the sorted bin (a bin-overflow tile,
        // which has no sorted bin, keeps its FP32 decisions)
        if constexpr (sizeof(T) == 4 && EXACT) {
            if (amb && count > 0 && count <= a.cap) {
                float gmv[3] = {0.0f, 0.0f, 0.0f};
                double zw;
                good = false;
                int gfv = -1;
                fac = pixel_posvis64(a, g, ids, count, li, lj, (double)pi * g.kmpp, (double)pj * g.kmpp, &zw,
                                     &good, gmv, &gfv);
                zz = (float)zw;
                zlo = (float)(zw - (double)zz);
                gfac = gfv; gm0 = gmv[0]; gm1 = gmv[1]; gm2 = gmv[2];
                gready = true;
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (good && !lcv && !gready) good_normal_f32(a, g, gfac, gsv, gtv, smooth, gm0, gm1, gm2);
        }

        // cos(e) / cos(i) of the last winner whose smoothed normal faced the
        // viewer: cotrans + normalize (posvis.c:250-274), once per pixel
        double ce64 = 0.0, ci64 = 0.0;      // lcv: the FP64 cosines
        if (good && lcv) {
            lc_cos64(a, g, gfac, (double)pi * g.kmpp, (double)pj * g.kmpp, smooth,
                     bistatic_obs, &ce64, &ci64);
            cosa = (T)ce64;
            cosb = (T)ci64;
        } else if (good) {
            T n0 = gm0, n1 = gm1, n2 = gm2;
            T oa[12];
            load_oa<T>(g, oa);
            if (smooth) {
                T r0 = 0, r1 = 0, r2 = 0;
                r0 += oa[0] * gm0; r0 += oa[1] * gm1; r0 += oa[2] * gm2;
                r1 += oa[3] * gm0; r1 += oa[4] * gm1; r1 += oa[5] * gm2;
                r2 += oa6 * gm0; r2 += oa7 * gm1; r2 += oa8 * gm2;
                T norm = 0;
                norm += r0 * r0; norm += r1 * r1; norm += r2 * r2;
                norm = sqrt(norm);
                if (norm != (T)0) { r0 /= norm; r1 /= norm; r2 /= norm; }
                n0 = r0; n1 = r1; n2 = r2;
            }
            if (n2 > (T)0) {
                cosa = n2;
                if (bistatic_obs) {
                    cosb = n0 * oa[9] + n1 * oa[10] + n2 * oa[11];
                    if (cosb <= (T)0) cosa = 0;
                }
            }
        }

        // ---- outputs of this tile
        bool covered = inframe && fac >= 0;
        // FP64 depth. FP32 form: a radar pixel takes its float-pair depth
        // (a few 1e-9 km, 1e-7 of a delay bin); a lightcurve view, and an
        // exact radar view whose maps are kept, recompute the winning facet's
        // depth in FP64 with the FP64 form's operations (facet_depth64),
        // because posmask's shadow test compares it with the sun view's to a
        // few 1e-8 km and the kept maps are the FP64 form's.
        double z64 = (double)zz;
        if constexpr (sizeof(T) == 4) {
            if (fac < 0) {
                z64 = -SHAPE_HUGENUMBER;
            } else if (g.kind != VIEW_RADAR || (EXACT && writes_pos)) {
                const double4 *vt = static_cast<const double4 *>(a.vt) + g.vt_base;
                z64 = facet_depth64(vt, a.fvi[fac], (double)pi * g.kmpp, (double)pj * g.kmpp);
            } else {
                z64 = (double)zz + (double)zlo;
            }
        }
        if (inframe && writes_pos) {
            long long p = g.pos_base + (long long)(pi + n) * g.side + (pj + n);
            double *Z = static_cast<double *>(a.pos_z);
            T *CE = static_cast<T *>(a.pos_cose), *CI = static_cast<T *>(a.pos_cosi);
            if constexpr (sizeof(T) == 8) {
                if (a.accumulate) {
                    // assigned by this launch: a win always changes the facet
                    // (the pixel was blank) or raises the depth
                    const bool won = (Z[p] != z64) || (a.pos_f[p] != fac);
                    a.won[p] = won ? 1 : 0;
                    covered = won;
                }
            }
            Z[p] = z64;
            a.pos_f[p] = fac;
            if (lcv) {                           // FP32 form, lightcurve views: FP64 cosines
                static_cast<double *>(a.pos_cose)[p] = ce64;
                if (g.kind != VIEW_LC_SUN) static_cast<double *>(a.pos_cosi)[p] = ci64;
            } else {
                CE[p] = cosa;                    // cos(e), or cos(i) in the sun view (pos->cosill)
                if (g.kind != VIEW_LC_SUN) CI[p] = cosb;
            }
        }
        // covered-pixel bbox (POSrect with (i,i,j,j), posvis.c:278-280)
        int cimin = covered ? pi : INT_MAX, cimax = covered ? pi : INT_MIN;
        int cjmin = covered ? pj : INT_MAX, cjmax = covered ? pj : INT_MIN;
        cimin = warp_min(cimin); cimax = warp_max(cimax);
        cjmin = warp_min(cjmin); cjmax = warp_max(cjmax);
        PixPos pp = {0.0, 0.0};
        bool lit = false;
        PixDD<T> dd;
        dd.ok = false;
        T scose = 0;
        if (g.kind == VIEW_RADAR && covered) {
            if (a.mark_seen && !g.no_seen && (double)cosa > a.mincosine_seen)
                a.seen[fac] = 1;
        }
        const DDC<T> kc = load_ddc<T>(g);
        if (g.kind == VIEW_RADAR) {
            // Synthesis runs on a permuted pixel-to-thread map: the replay
            // wants each warp on a compact 4x8 block, but neighbouring pixels
            // hit the same delay-Doppler bins, so a compact warp's atomics
            // would repeat addresses within one instruction; a warp of
            // scattered pixels rarely does.
            const int me = li * TILE_W + lj;
            s_pz[me] = z64;
            s_pc[me] = (covered && cosa > (T)0) ? cosa : (T)0;
            __syncthreads();
            const int q = (tid * 37 + 11) & (TILE_PIX - 1);
            scose = s_pc[q];
            if (scose > (T)0) {
                lit = true;
                if constexpr (sizeof(T) == 4)
                    dd = pixel_dd_setup_x(g, ti0 + q / TILE_W, tj0 + q % TILE_W, s_pz[q], pp);
                else
                    dd = pixel_dd_setup<T>(g, kc, ti0 + q / TILE_W, tj0 + q % TILE_W, s_pz[q], pp);
            }
        }
        if (lane == 0) {
            s_red[wid][0] = cimin; s_red[wid][1] = cimax; s_red[wid][2] = cjmin; s_red[wid][3] = cjmax;
        }
        // (reduced before the scatter, so the positions are not live across it)
        if (g.kind == VIEW_RADAR) {
            // delay / Doppler extremes of the lit pixels as dkey keys (unlit
            // lanes hold the neutral key)
            const unsigned long long kd = dkey(pp.del), kp = dkey(pp.dop);
            const unsigned long long k0 = warp_kmin(lit ? kd : ~0ull), k1 = warp_kmax(lit ? kd : 0ull);
            const unsigned long long k2 = warp_kmin(lit ? kp : ~0ull), k3 = warp_kmax(lit ? kp : 0ull);
            if (lane == 0) {
                s_redk[wid][0] = k0; s_redk[wid][1] = k1; s_redk[wid][2] = k2; s_redk[wid][3] = k3;
            }
        }
        // The footprint goes straight to the frame's fit image in HBM: FP32 as
        // 16-byte vector reductions, FP64 as scalar atomics (both measured
        // faster than a shared-memory accumulator flushed per tile).
        if (g.kind == VIEW_RADAR && dd.ok) {
            if constexpr (sizeof(T) == 4) {
                if (g.dop1d) pixel_dop_scatter_f32_64(a, g, kc, scose, dd);
                else pixel_dd_scatter_f32_direct(a, g, kc, scose, dd, static_cast<float *>(a.fit) + g.fit_base);
            } else
                pixel_dd_scatter<T>(a, g, kc, scose, dd, static_cast<T *>(a.fit) + g.fit_base, 1, 1, g.ndop);
        } else if (g.kind == VIEW_RADAR && g.dop1d && lit) {
            a.states[item.x].any_overflow = 1;
            pixel_dop_overflow<T>(a, g, kc, scose, dd);
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
                unsigned long long k0 = ~0ull, k1 = 0ull, k2 = ~0ull, k3 = 0ull;
                for (int ww = 0; ww < RASTER_THREADS / 32; ww++) {
                    k0 = min(k0, s_redk[ww][0]); k1 = max(k1, s_redk[ww][1]);
                    k2 = min(k2, s_redk[ww][2]); k3 = max(k3, s_redk[ww][3]);
                }
                if (k0 != ~0ull) {        // a lit pixel in the tile
                    int l[4];
                    dd_bin_limits(g, dkey_inv(k0), dkey_inv(k1), dkey_inv(k2), dkey_inv(k3), l);
                    atomicMin(&S.idellim[0], l[0]); atomicMax(&S.idellim[1], l[1]);
                    atomicMin(&S.idoplim[0], l[2]); atomicMax(&S.idoplim[1], l[3]);
                    atomicMin(&S.dellim[0], k0); atomicMax(&S.dellim[1], k1);
                    atomicMin(&S.doplim[0], k2); atomicMax(&S.doplim[1], k3);
                    S.any_lit = 1;
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------
// Warp-independent tile raster. The CTA still takes one 16x16 tile (its bin
// read once into L1), but each of its 8 warps works its 4x8 block on its own,
// with no CTA-wide barrier: a warp collects the bin's facets whose bbox
// meets its block, sorts them by facet index, stages and replays them 32 at
// a time, then finalizes, writes and scatters its own 32 pixels and moves
// the frame limits with atomics it skips when they cannot change anything.
// Blocks of one tile differ in work by about 2x on average, so the CTA-wide
// barriers of k_raster kept the faster warps of a tile idle.
constexpr int WARP_LIST = 128;       // facets a warp block sorts in shared memory

template <typename T>
struct WarpArea {
    int2 ids[WARP_LIST];             // the block's bin entries, in facet order
    Stage<T> st[32];                 // the chunk being replayed
};

template <typename T, bool EXACT>
__global__ void __launch_bounds__(RASTER_THREADS, sizeof(T) == 8 ? RASTER_W_MIN_BLOCKS_F64 : RASTER_W_MIN_BLOCKS)
k_raster_w(RasterArgs a)
{
    grid_dep_wait();
    extern __shared__ __align__(32) unsigned char smem[];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    WarpArea<T> &wa = reinterpret_cast<WarpArea<T> *>(smem)[wid];
    int2 *ids = wa.ids;
    Stage<T> *st = wa.st;
    const unsigned lt_mask = (1u << lane) - 1u;
    // warp wid owns a 4x8 block of the 16x16 tile
    const int bi0 = 4 * (wid >> 1), bj0 = 8 * (wid & 1);
    const int li = bi0 + (lane >> 3), lj = bj0 + (lane & 7);

    for (int w = blockIdx.x; w < a.nwork; w += gridDim.x) {
        const int2 item = a.work[w];
        const FrameGeom &g = a.geoms[item.x];
        const int tile = item.y;
        const int tx = tile / g.tiles_x, ty = tile % g.tiles_x;
        const int n = g.n;
        const int ti0 = -n + tx * TILE_W, tj0 = -n + ty * TILE_W;
        const int ti1 = min(ti0 + TILE_W - 1, n), tj1 = min(tj0 + TILE_W - 1, n);
        const int pi = ti0 + li, pj = tj0 + lj;
        const bool inframe = (pi <= n) && (pj <= n);
        const int count = a.bin_count[g.tile_base + tile];
        const bool writes_pos = (g.kind != VIEW_RADAR) || a.keep_pos;
        if (count == 0 && !writes_pos) continue;
        // a block wholly outside the frame (the tile's last rows or columns)
        if (bi0 > ti1 - ti0 || bj0 > tj1 - tj0) continue;

        const double ox = (double)ti0 * g.kmpp, oy = (double)tj0 * g.kmpp;
        const T x0 = (sizeof(T) == 8) ? (T)pi * (T)g.kmpp : (T)((double)li * g.kmpp);
        const T x1 = (sizeof(T) == 8) ? (T)pj * (T)g.kmpp : (T)((double)lj * g.kmpp);
        T zz = (T)(-SHAPE_HUGENUMBER), cosa = 0, cosb = 0;
        int fac = -1;
        if constexpr (sizeof(T) == 8) {
            if (a.accumulate && inframe) {
                const long long p = g.pos_base + (long long)(pi + n) * g.side + (pj + n);
                zz = static_cast<const double *>(a.pos_z)[p];
                fac = a.pos_f[p];
                cosa = static_cast<const T *>(a.pos_cose)[p];
                if (g.kind != VIEW_LC_SUN) cosb = static_cast<const T *>(a.pos_cosi)[p];
            }
        }
        T zze = 0, zlo = 0;
        bool amb = false, good = false;
        T gm0 = 0, gm1 = 0, gm2 = 0;
        int gfac = -1;
        float gsv = 0.0f, gtv = 0.0f;
        bool gready = false;
        const bool smooth = g.smooth != 0;
        const bool bistatic_obs = (g.kind == VIEW_LC_OBS);
        const T oa6 = (T)g.oa[6], oa7 = (T)g.oa[7], oa8 = (T)g.oa[8];
        const unsigned pxw = pack_px(li, lj);
        auto visit = [&](const Stage<T> &s) {
            T sv, tv, z, zr = 0;
            if constexpr (sizeof(T) == 8) {
                if (__vcmpgeu4(pxw, s.bb) != 0xffffffffu) return;
                const auto p0 = s.p0, p1 = s.p1;
                const T dx = x0 - p0.x, dy = x1 - p0.y;
                sv = (dx * p0.z - p0.w * dy) * p1.x;
                if (!((sv >= (T)-SHAPE_SMALLVAL) && (sv <= (T)1.0 + (T)SHAPE_SMALLVAL))) return;
                tv = (p1.y * dy - dx * p1.z) * p1.x;
                if (!((tv >= (T)-SHAPE_SMALLVAL) && (tv <= sv + (T)SHAPE_SMALLVAL))) return;
                const auto p2 = s.p2;
                z = p1.w + sv * p2.x + tv * p2.y;
                if (!((z > zz) || (fac < 0))) return;
            } else {
                const auto p0 = s.p0, p1 = s.p1, p2 = s.p2;
                const float4 be = *reinterpret_cast<const float4 *>(&s.bb);
                const bool inb = __vcmpgeu4(pxw, __float_as_uint(be.x)) == 0xffffffffu;
                const T dx = x0 - p0.x, dy = x1 - p0.y;
                sv = fmaf(p0.z, dx, p0.w * dy);
                tv = fmaf(p1.x, dx, p1.y * dy);
                zr = fmaf(p1.z, dx, p1.w * dy);
                z = p2.y + zr;
                const T es = be.y, et = be.z, est = es + et;
                if constexpr (EXACT) {
                    const bool out = !inb || (sv < -2 * es) || (sv > 1 + 2 * es) || (tv < -2 * et) ||
                                     (tv > sv + 2 * est);
                    if (out) return;
                    const bool sure = (sv >= es) && (sv <= 1 - es) && (tv >= et) && (tv <= sv - est);
                    const bool near = (fac >= 0) && (fabsf(z - zz) <= be.w + zze);
                    amb = amb || !sure || near;
                    if (!((z > zz) || (fac < 0))) return;
                    zze = be.w;
                } else {
                    const bool in = inb && (sv >= (T)-SHAPE_SMALLVAL) && (sv <= (T)1.0 + (T)SHAPE_SMALLVAL) &&
                                    (tv >= (T)-SHAPE_SMALLVAL) && (tv <= sv + (T)SHAPE_SMALLVAL);
                    if (!(in && ((z > zz) || (fac < 0)))) return;
                }
            }
            const auto p2 = s.p2;
            zz = z;
            fac = s.f;
            if constexpr (sizeof(T) == 4) {
                const float bv = z - p2.y;
                zlo = ((p2.y - (z - bv)) + (zr - bv)) + p2.x;
            }
            if constexpr (sizeof(T) == 4) {
                // FP32: the sign from the staged linear form (as k_raster)
                if (smooth) {
                    const T r2 = s.q[0] + sv * s.q[1] + tv * s.q[2];
                    if constexpr (EXACT) amb = amb || (fabsf(r2) <= 4 * (s.es + s.et) + 3e-6f);
                    if (r2 > (T)0) { good = true; gfac = s.f; gsv = sv; gtv = tv; }
                } else {
                    good = true; gfac = s.f;
                }
            } else if (smooth) {
                const T m0 = s.q[0] + sv * (s.q[3] - s.q[0]) + tv * (s.q[6] - s.q[3]);
                const T m1 = s.q[1] + sv * (s.q[4] - s.q[1]) + tv * (s.q[7] - s.q[4]);
                const T m2 = s.q[2] + sv * (s.q[5] - s.q[2]) + tv * (s.q[8] - s.q[5]);
                T r2 = 0;
                r2 += oa6 * m0; r2 += oa7 * m1; r2 += oa8 * m2;
                if (r2 > (T)0) { good = true; gm0 = m0; gm1 = m1; gm2 = m2; }
            } else {
                good = true; gm0 = p2.z; gm1 = p2.w; gm2 = s.nz;
            }
        };

        // the block's facets: bin entries whose tile bbox meets the block
        int nb = 0;
        bool listed = (count > 0 && count <= a.cap);
        if (listed) {
            const int2 *bin = a.bin_ids + (size_t)(g.tile_base + tile) * a.cap;
            for (int base = 0; base < count; base += 32) {
                const int k = base + lane;
                int2 e = make_int2(0, 0);
                bool hit = false;
                if (k < count) {
                    e = bin[k];
                    const int b = e.y;
                    hit = (b & 15) <= bi0 + 3 && ((b >> 4) & 15) >= bi0 && ((b >> 8) & 15) <= bj0 + 7 &&
                          ((b >> 12) & 15) >= bj0;
                }
                const unsigned m = __ballot_sync(0xffffffffu, hit);
                const int pos = nb + __popc(m & lt_mask);
                if (hit && pos < WARP_LIST) ids[pos] = e;
                nb += __popc(m);
            }
            __syncwarp();
            listed = nb <= WARP_LIST;
        }
        if (listed && nb > 0) {
            // facet order (posvis walks facets in index order): a facet's rank
            // is the number of listed facets with a smaller index
            int2 mine[WARP_LIST / 32];
            int rank[WARP_LIST / 32];
#pragma unroll
            for (int r = 0; r < WARP_LIST / 32; r++) {
                const int k = lane + 32 * r;
                rank[r] = -1;
                if (k < nb) {
                    mine[r] = ids[k];
                    int c = 0;
                    for (int j = 0; j < nb; j++) c += (ids[j].x < mine[r].x);
                    rank[r] = c;
                }
            }
            __syncwarp();
#pragma unroll
            for (int r = 0; r < WARP_LIST / 32; r++)
                if (rank[r] >= 0) ids[rank[r]] = mine[r];
            __syncwarp();
            for (int c0 = 0; c0 < nb; c0 += 32) {
                const int nst = min(32, nb - c0);
                if (lane < nst) {
                    const int2 e = ids[c0 + lane];
                    Stage<T> sf;
                    const int bb = e.y;
                    sf.bb = pack_bb(bb & 15, (bb >> 4) & 15, (bb >> 8) & 15, (bb >> 12) & 15);
                    sf.wmask = 0;
                    stage_fill<T>(a, g, e.x, sf, ox, oy);
                    st[lane] = sf;
                }
                __syncwarp();
                for (int b = 0; b < nst; b++) visit(st[b]);
                __syncwarp();
            }
        } else if (count > 0 && !listed) {
            // bin or block list overflow: every facet of the model in index
            // order, keeping those that overlap this tile
            for (int c0 = 0; c0 < a.nf; c0 += 32) {
                Stage<T> sf;
                bool ok = false;
                if (c0 + lane < a.nf) ok = stage_facet<T>(a, g, c0 + lane, ti0, ti1, tj0, tj1, sf, ox, oy);
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) st[__popc(bal & lt_mask)] = sf;
                __syncwarp();
                const int tot = __popc(bal);
                for (int b = 0; b < tot; b++) visit(st[b]);
                __syncwarp();
            }
        }

        // FP32 form: a pixel with a decision within FP32 error is redone by
        // the FP64 form's rules over the block's sorted list (an overflowing
        // block, which has none, keeps its FP32 decisions)
        if constexpr (sizeof(T) == 4 && EXACT) {
            if (amb && listed && nb > 0) {
                float gmv[3] = {0.0f, 0.0f, 0.0f};
                double zw;
                good = false;
                int gfv = -1;
                fac = pixel_posvis64(a, g, ids, nb, li, lj, (double)pi * g.kmpp, (double)pj * g.kmpp, &zw, &good,
                                     gmv, &gfv);
                zz = (float)zw;
                zlo = (float)(zw - (double)zz);
                gfac = gfv; gm0 = gmv[0]; gm1 = gmv[1]; gm2 = gmv[2];
                gready = true;
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (good && !gready) good_normal_f32(a, g, gfac, gsv, gtv, smooth, gm0, gm1, gm2);
        }

        if (good) {
            T n0 = gm0, n1 = gm1, n2 = gm2;
            T oa[12];
            load_oa<T>(g, oa);
            if (smooth) {
                T r0 = 0, r1 = 0, r2 = 0;
                r0 += oa[0] * gm0; r0 += oa[1] * gm1; r0 += oa[2] * gm2;
                r1 += oa[3] * gm0; r1 += oa[4] * gm1; r1 += oa[5] * gm2;
                r2 += oa6 * gm0; r2 += oa7 * gm1; r2 += oa8 * gm2;
                T norm = 0;
                norm += r0 * r0; norm += r1 * r1; norm += r2 * r2;
                norm = sqrt(norm);
                if (norm != (T)0) { r0 /= norm; r1 /= norm; r2 /= norm; }
                n0 = r0; n1 = r1; n2 = r2;
            }
            if (n2 > (T)0) {
                cosa = n2;
                if (bistatic_obs) {
                    cosb = n0 * oa[9] + n1 * oa[10] + n2 * oa[11];
                    if (cosb <= (T)0) cosa = 0;
                }
            }
        }

        bool covered = inframe && fac >= 0;
        double z64 = (double)zz;
        if constexpr (sizeof(T) == 4) {
            if (fac < 0) {
                z64 = -SHAPE_HUGENUMBER;
            } else if (g.kind != VIEW_RADAR || (EXACT && writes_pos)) {
                const double4 *vt = static_cast<const double4 *>(a.vt) + g.vt_base;
                z64 = facet_depth64(vt, a.fvi[fac], (double)pi * g.kmpp, (double)pj * g.kmpp);
            } else {
                z64 = (double)zz + (double)zlo;
            }
        }
        if (inframe && writes_pos) {
            long long p = g.pos_base + (long long)(pi + n) * g.side + (pj + n);
            double *Z = static_cast<double *>(a.pos_z);
            T *CE = static_cast<T *>(a.pos_cose), *CI = static_cast<T *>(a.pos_cosi);
            if constexpr (sizeof(T) == 8) {
                if (a.accumulate) {
                    const bool won = (Z[p] != z64) || (a.pos_f[p] != fac);
                    a.won[p] = won ? 1 : 0;
                    covered = won;
                }
            }
            Z[p] = z64;
            a.pos_f[p] = fac;
            CE[p] = cosa;
            if (g.kind != VIEW_LC_SUN) CI[p] = cosb;
        }
        FrameState &S = a.states[item.x];
        // covered-pixel bbox (POSrect with (i,i,j,j), posvis.c:278-280); an
        // atomic only where it can move the frame's value
        {
            const int cimin = warp_min(covered ? pi : INT_MAX), cimax = warp_max(covered ? pi : INT_MIN);
            const int cjmin = warp_min(covered ? pj : INT_MAX), cjmax = warp_max(covered ? pj : INT_MIN);
            if (lane == 0 && cimin != INT_MAX) {
                if (cimin < *(volatile int *)&S.cov_i[0]) atomicMin(&S.cov_i[0], cimin);
                if (cimax > *(volatile int *)&S.cov_i[1]) atomicMax(&S.cov_i[1], cimax);
                if (cjmin < *(volatile int *)&S.cov_j[0]) atomicMin(&S.cov_j[0], cjmin);
                if (cjmax > *(volatile int *)&S.cov_j[1]) atomicMax(&S.cov_j[1], cjmax);
            }
        }
        if (g.kind == VIEW_RADAR) {
            if (covered && a.mark_seen && !g.no_seen && (double)cosa > a.mincosine_seen) a.seen[fac] = 1;
            const DDC<T> kc = load_ddc<T>(g);
            PixPos pp = {0.0, 0.0};
            PixDD<T> dd;
            dd.ok = false;
            const bool lit = covered && cosa > (T)0;
            if (lit) {
                if constexpr (sizeof(T) == 4)
                    dd = pixel_dd_setup_x(g, pi, pj, z64, pp);
                else
                    dd = pixel_dd_setup<T>(g, kc, pi, pj, z64, pp);
            }
            // delay / Doppler extremes of the lit pixels as dkey keys
            const unsigned long long kd = dkey(pp.del), kp = dkey(pp.dop);
            const unsigned long long k0 = warp_kmin(lit ? kd : ~0ull), k1 = warp_kmax(lit ? kd : 0ull);
            const unsigned long long k2 = warp_kmin(lit ? kp : ~0ull), k3 = warp_kmax(lit ? kp : 0ull);
            if (lane == 0 && k0 != ~0ull) {
                int l[4];
                dd_bin_limits(g, dkey_inv(k0), dkey_inv(k1), dkey_inv(k2), dkey_inv(k3), l);
                if (l[0] < *(volatile int *)&S.idellim[0]) atomicMin(&S.idellim[0], l[0]);
                if (l[1] > *(volatile int *)&S.idellim[1]) atomicMax(&S.idellim[1], l[1]);
                if (l[2] < *(volatile int *)&S.idoplim[0]) atomicMin(&S.idoplim[0], l[2]);
                if (l[3] > *(volatile int *)&S.idoplim[1]) atomicMax(&S.idoplim[1], l[3]);
                if (k0 < *(volatile unsigned long long *)&S.dellim[0]) atomicMin(&S.dellim[0], k0);
                if (k1 > *(volatile unsigned long long *)&S.dellim[1]) atomicMax(&S.dellim[1], k1);
                if (k2 < *(volatile unsigned long long *)&S.doplim[0]) atomicMin(&S.doplim[0], k2);
                if (k3 > *(volatile unsigned long long *)&S.doplim[1]) atomicMax(&S.doplim[1], k3);
                if (!*(volatile int *)&S.any_lit) S.any_lit = 1;
            }
            if (dd.ok) {
                if constexpr (sizeof(T) == 4) {
                    if (g.dop1d) pixel_dop_scatter_f32_64(a, g, kc, cosa, dd);
                    else pixel_dd_scatter_f32_direct(a, g, kc, cosa, dd, static_cast<float *>(a.fit) + g.fit_base);
                } else
                    pixel_dd_scatter<T>(a, g, kc, cosa, dd, static_cast<T *>(a.fit) + g.fit_base, 1, 1, g.ndop);
            } else if (g.dop1d && lit) {
                S.any_overflow = 1;
                pixel_dop_overflow<T>(a, g, kc, cosa, dd);
            }
        }
        __syncwarp();
    }
}

// Dynamic shared memory of a raster CTA: the ranked bin, then the staging
// area, large enough for the staged facets and for the rank's scratch (the
// bitmap and prefix counts, 8 bytes per 32 facets, plus the raw bin).
template <typename T>
inline size_t raster_smem_bytes(int cap, int nf)
{
    const size_t nw = ((size_t)nf + 31) / 32;
    const size_t fused = nw <= (size_t)FUSED_RANK_MAX_WORDS ? 8 * nw : 0;
    return raster_ids_bytes(cap) + raster_stage_bytes<T>(cap, nf) + fused;
}

// Called once per device before any launch (not inside stream capture).
// Both kernels run several CTAs per SM, which needs the largest
// shared-memory carveout.
template <typename T, bool EXACT>
inline cudaError_t configure_raster_one()
{
    cudaError_t e = cudaFuncSetAttribute(k_raster<T, EXACT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_raster<T, EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_raster_w<T, EXACT>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_raster_w<T, EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(RASTER_THREADS / 32 * sizeof(WarpArea<T>)));
    return e;
}
template <typename T>
inline cudaError_t configure_raster_t()
{
    cudaError_t e = configure_raster_one<T, false>();
    if (e != cudaSuccess || sizeof(T) == 8) return e;
    e = configure_raster_one<T, true>();
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_raster<T, true, true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_raster<T, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    return e;
}

template <typename T>
inline void launch_raster_t(const RasterArgs &a, cudaStream_t s)
{
    if (a.nwork <= 0) return;
    RasterArgs b = a;
    const int grid = (a.grid > 0 && a.grid < a.nwork) ? a.grid : a.nwork;
    // the FP64 form is exact by construction; the FP32 form runs its exact
    // variant unless radar views are asked for their FP32 decisions
    if (a.variant == 1) {
        b.smem_bytes = RASTER_THREADS / 32 * sizeof(WarpArea<T>);
        if (sizeof(T) == 4 && a.exact)
            launch_k(k_raster_w<T, true>, dim3(grid), dim3(RASTER_THREADS), b.smem_bytes, s, a.pdl != 0, b);
        else
            launch_k(k_raster_w<T, false>, dim3(grid), dim3(RASTER_THREADS), b.smem_bytes, s, a.pdl != 0, b);
        return;
    }
    b.smem_bytes = raster_smem_bytes<T>(a.cap, a.nf);
    if (sizeof(T) == 4 && a.exact && a.lc_views)
        launch_k(k_raster<T, true, true>, dim3(grid), dim3(RASTER_THREADS), b.smem_bytes, s, a.pdl != 0, b);
    else if (sizeof(T) == 4 && a.exact)
        launch_k(k_raster<T, true>, dim3(grid), dim3(RASTER_THREADS), b.smem_bytes, s, a.pdl != 0, b);
    else
        launch_k(k_raster<T, false>, dim3(grid), dim3(RASTER_THREADS), b.smem_bytes, s, a.pdl != 0, b);
}

// Resident CTAs per SM of the kernel launch_raster_t would launch for a
// (0 when the query fails): the persistent grid is this times the SM count.
template <typename T>
inline int raster_occupancy_t(const RasterArgs &a)
{
    int n = 0;
    cudaError_t e;
    if (a.variant == 1) {
        const size_t sm = RASTER_THREADS / 32 * sizeof(WarpArea<T>);
        e = (sizeof(T) == 4 && a.exact)
                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_raster_w<T, true>, RASTER_THREADS, sm)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_raster_w<T, false>, RASTER_THREADS, sm);
    } else {
        const size_t sm = raster_smem_bytes<T>(a.cap, a.nf);
        e = (sizeof(T) == 4 && a.exact && a.lc_views)
                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_raster<T, true, true>, RASTER_THREADS, sm)
            : (sizeof(T) == 4 && a.exact)
                ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_raster<T, true>, RASTER_THREADS, sm)
                : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_raster<T, false>, RASTER_THREADS, sm);
    }
    return e == cudaSuccess ? n : 0;
}

}  // namespace shape
