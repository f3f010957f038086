// Internal device-side data layout of the SHAPE B200 engine.
//
// HBM layout (all frames of all datasets of one engine live in flat arenas):
//   model     : vparam (a,u as double3 x nv, r[nv], scale[3]) -> realized
//               vx/vn as double4[nv] (one 32-byte load per vertex), fn as
//               double4[nf], fvi as int4[nf] (corner indices + pad)
//   per frame : FrameGeom (constants, read-only), FrameState (atomics,
//               reset every evaluation), transformed vertices vt
//               (T4[nv] per frame view), facet bins (TILE_CAP ids per
//               16x16 POS tile), fit image (T, ndel*ndop), obs and
//               1/variance (double, ndel*ndop)
//   per lightcurve point: two FrameGeom views (observer, sun) and POS maps
//               z/cose/cosi/f plus zill/fill that posmask reads.
#pragma once

#include <cstdint>

#include "shape_types.h"

namespace shape {

constexpr int TILE_W = 16;          // POS tile: 16 x 16 pixels, one CTA
constexpr int TILE_PIX = TILE_W * TILE_W;
constexpr int RASTER_THREADS = TILE_PIX;
constexpr int STAGE_FACETS = 128;   // facets staged in shared memory per pass
constexpr int CHI2_THREADS = 256;
constexpr int CHI2_LANE = 16;       // bins per lane of a chi-square item
constexpr int CHI2_ITEM = 32 * CHI2_LANE;   // bins per item: one warp's
constexpr int FIT32_PAD = 16;       // FP32 fit arena padding (vector reductions, k_raster)
constexpr int DOP_MAXOVERFLOW = 2000;   // Doppler overflow spectrum bins (MAXOVERFLOW, src/shape/const.h:181)

// View kinds of a FrameGeom.
constexpr int VIEW_RADAR = 0;       // delay-Doppler frame, observer view
constexpr int VIEW_LC_OBS = 1;      // lightcurve point, observer view (bistatic)
constexpr int VIEW_LC_SUN = 2;      // lightcurve point, sun view (src = 1)
constexpr int VIEW_POS = 3;         // a plane-of-sky view of its own (monostatic observer view, no synthesis)

struct FrameGeom {
    double oa[9];        // observer(or sun) <- body, row-major, reference op order
    double usrc[3];      // sun direction in observer coords (VIEW_LC_OBS)
    double off[3];       // orbit offset added to the view-frame vertices (posvis's orbit_offset; 0 here otherwise)
    double wscale;       // weight of this view's cross-section in its frame: 1 / views of a smeared frame
    int no_seen;         // 1: a smeared frame's view other than the frame's epoch view (marks no seen facets)
    double kmpp;
    int n, side;         // POS half width, 2n+1
    int tiles_x;         // tiles per POS side
    int tile_base;       // first tile of this view in the tile arrays
    int vt_base;         // first transformed vertex (view * nv)
    int kind;            // VIEW_*
    int smooth;          // pos_smooth for this view
    int ndel, ndop;      // delay-Doppler size (VIEW_RADAR)
    long long pos_base;  // offset of this view's POS maps (keep_pos / lightcurves)
    long long fit_base;  // offset of this frame's image in fit/obs/oov
    // pos2deldop constants (src/shape/pos2deldop.c:218-275), computed on the host
    double delfact, delshift, ax, ay, dopshift, const1, const2, one_over_spb;
    double xincr, yincr, dopdiff_bl, dopdiff_max, dopDC_vig, dopfftlen;
    int codemethod, spb, stride, spb_over_stride, spb_sq, nsinc2, nsinc2_sq, sinc2width;
    int law;             // index into the radar law table
    int frame_index;     // global radar frame index or lightcurve point index
    // Doppler-only frames run as one-row delay-Doppler frames whose delay
    // response is exactly 1; pixels whose footprint leaves the spectrum go to
    // an overflow spectrum of DOP_MAXOVERFLOW bins (src/shape/pos2doppler.c)
    int dop1d;           // 1: Doppler spectrum
    int idop0;           // overflow bin of spectrum bin 0: MAXOVERFLOW/2 - floor(dopshift + 0.5)
    long long ovf_base;  // first element of this frame's overflow spectrum
    // the synthesis constants rounded to float on the host for the FP32
    // raster, in FDD_* order (five float4 loads per tile instead of one
    // double->float conversion per constant per pixel)
    alignas(16) float fdd[20];
    alignas(16) float foa[12];   // oa[9] and usrc[3] rounded to float
};

// Order of FrameGeom::fdd.
enum {
    FDD_DELFACT, FDD_DELSHIFT, FDD_AX, FDD_AY, FDD_DOPSHIFT, FDD_CONST1, FDD_CONST2, FDD_ONE_OVER_SPB,
    FDD_XINCR, FDD_YINCR, FDD_DOPDIFF_BL, FDD_DOPDIFF_MAX, FDD_DOPDC_VIG, FDD_DOPFFTLEN, FDD_KMPP,
    FDD_HALF_W, FDD_SPB_OVER_STRIDE, FDD_STRIDE, FDD_SPB_SQ, FDD_NSINC2_SQ, FDD_N
};

// Per-view accumulators, reset by k_reset_state each evaluation.
struct FrameState {
    int outbnd;
    int bin_overflow;
    int cov_i[2], cov_j[2];          // covered-pixel bbox (min i, max i), (min j, max j)
    int ofr_i[2], ofr_j[2];          // POSrect updates of facets wholly outside the frame
    unsigned long long ofr_ov[4];    // ordered keys: imin, imax, jmin, jmax (doubles)
    int idellim[2], idoplim[2];
    unsigned long long dellim[2], doplim[2];  // ordered keys of min / max
    int any_lit;
    int any_overflow;                // Doppler frame: a footprint left the spectrum
};

// Radar scattering law table entry (mirror of shape_radar_law).
struct RadarLawDev {
    int type;
    double diff_R, diff_C, qs_R, qs_C, qs_cos_cutoff;
    int diff_linear, qs_linear;   // 2C - 1 == 1: cos^(2C-1) is cos itself
};

// Lightcurve point descriptor (one calc epoch).
struct LcPointDev {
    double so[9];             // sun <- observer: se * oe^T (src/shape/posmask.c:70-71)
    int obs_view, sun_view;   // FrameGeom indices
    int set;                  // lightcurve set index
    int law_type;             // SHAPE_OPTLAW_*
    double intensityfactor;   // (kmpp/AU)^2 (src/shape/calc_fits.c:1714)
    double s_ls, s_l, scale;  // law constants (apply_photo.c:85-133, 226-248)
    double mask_tol;
    double pixels_per_km;     // 1/kmpp
    long long b_base;         // plane-of-sky frame: offset of its brightness image (-1: a lightcurve point)
};

// Plane-of-sky frame descriptor (calc_poset's resampling and chi2_poset).
struct PosetFrameDev {
    int point;                // its LcPointDev (observer and sun views, brightness image)
    int ncol, nrow;
    long long img_base;       // offset of its fit / observed / 1/variance images
    double x0, xwidth, y0, ywidth;    // resampim's grid (src/shape/calc_fits.c:1278-1287)
    double cosang, sinang;    // cos and sin of the grid rotation (-northangle), from the C library
    int mode, rebin;          // SHAPE_RESAMPLE_*, image_rebin
    double weight, dof;
};

// Order-preserving 64-bit key of a double (for atomicMin/atomicMax).
__host__ __device__ inline unsigned long long dkey(double d)
{
    unsigned long long b;
#ifdef __CUDA_ARCH__
    b = (unsigned long long)__double_as_longlong(d);
#else
    __builtin_memcpy(&b, &d, 8);
#endif
    return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__host__ __device__ inline double dkey_inv(unsigned long long k)
{
    unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffULL) : ~k;
    double d;
#ifdef __CUDA_ARCH__
    d = __longlong_as_double((long long)b);
#else
    __builtin_memcpy(&d, &b, 8);
#endif
    return d;
}

}  // namespace shape
