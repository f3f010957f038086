// FP64 core kernels of the SHAPE B200 engine: model realization, view
// transforms, facet binning, chi-square reductions, lightcurve photometry
// and the evaluation summary.
//
// This translation unit is compiled with -fmad=false: the realization, the
// view transforms and the facet bounding boxes must reproduce the reference
// CPU arithmetic bit for bit (no a*b+c contraction), because they decide
// which POS pixels each facet covers. Expressions keep the reference's
// association order; sums that the reference starts from a literal 0.0
// (cotrans, src/util/cotrans.c; mmmul) start from 0.0 here as well.
#include <cfloat>
#include <climits>

#include "kernels.h"
#include "posmask_dev.cuh"

namespace shape {

namespace {

constexpr double SMALLVAL = SHAPE_SMALLVAL;
constexpr double HUGENUMBER = SHAPE_HUGENUMBER;

__device__ inline double dmin_(double a, double b) { return (a < b) ? a : b; }
__device__ inline double dmax_(double a, double b) { return (a > b) ? a : b; }
__device__ inline int clamp_lo(double v) { return (v < (double)INT_MIN) ? INT_MIN : (int)v; }
__device__ inline int clamp_hi(double v) { return (v > (double)INT_MAX) ? INT_MAX : (int)v; }

// ---------------------------------------------------------------- realize

// x = scale * (u*r + a)  (src/shape/realize_mod.c:471-479)
// Several components (vcomp and cxf non-null): vertex i takes its
// component's scale factors, then the component's rotation (comp.m, when
// its rotation offsets are not all zero) and translation (when its offsets
// are not all zero), as realize_mod does (src/shape/realize_mod.c:474-512).
// cxf holds per component m (9, row-major), off (3) and the two flags.
__device__ inline double4 realize_vertex(int i, const double *__restrict__ a, const double *__restrict__ u,
                                         const double *__restrict__ r, const double *__restrict__ scale,
                                         const int *__restrict__ vcomp, const double *__restrict__ cxf)
{
    const int c = vcomp ? vcomp[i] : 0;
    const double *sc = scale + 3 * c;
    double ri = r[i];
    double x0 = sc[0] * (u[3 * i + 0] * ri + a[3 * i + 0]);
    double x1 = sc[1] * (u[3 * i + 1] * ri + a[3 * i + 1]);
    double x2 = sc[2] * (u[3 * i + 2] * ri + a[3 * i + 2]);
    if (cxf) {
        const double *T = cxf + CXF_N * c;
        if (T[12] != 0.0) {
            double y[3];
            for (int j = 0; j < 3; j++) {
                y[j] = 0.0;
                y[j] += T[3 * j + 0] * x0;
                y[j] += T[3 * j + 1] * x1;
                y[j] += T[3 * j + 2] * x2;
            }
            x0 = y[0]; x1 = y[1]; x2 = y[2];
        }
        if (T[13] != 0.0) {
            x0 += T[9]; x1 += T[10]; x2 += T[11];
        }
    }
    return make_double4(x0, x1, x2, 0.0);
}

// facet normal and area: facnrm (src/shape/facnrm.c:13-25), cross
// (src/util/cross.c), normalize (src/util/normalize.c)
__device__ inline void realize_facet(int f, const int *__restrict__ fv, double4 p0, double4 p1, double4 p2,
                                     double4 *__restrict__ fn, double *__restrict__ area)
{
    double a0 = p1.x - p0.x, a1 = p1.y - p0.y, a2 = p1.z - p0.z;
    double b0 = p2.x - p1.x, b1 = p2.y - p1.y, b2 = p2.z - p1.z;
    double c0 = a1 * b2 - a2 * b1;
    double c1 = a2 * b0 - a0 * b2;
    double c2 = a0 * b1 - a1 * b0;
    area[f] = 0.5 * sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    double norm = 0.0;
    norm += c0 * c0;
    norm += c1 * c1;
    norm += c2 * c2;
    norm = sqrt(norm);
    if (norm != 0.0) {
        c0 /= norm; c1 /= norm; c2 /= norm;
    }
    fn[f] = make_double4(c0, c1, c2, 0.0);
}

// Vertices and facets in one launch: threads [0, nf) realize a facet from
// its three corners, which they compute themselves with the vertex formula
// (same operations, so the same bits as the vertex threads), and threads
// [nf, nf + nv) realize the vertices for the later stages.
__global__ void k_realize_vf(int nv, int nf, const double *__restrict__ a, const double *__restrict__ u,
                             const double *__restrict__ r, const double *__restrict__ scale,
                             const int *__restrict__ vcomp, const double *__restrict__ cxf,
                             const int *__restrict__ fv, double4 *__restrict__ vx, double4 *__restrict__ fn,
                             double *__restrict__ area, int4 *__restrict__ fvi)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < nf) {
        int i0 = fv[3 * k + 0], i1 = fv[3 * k + 1], i2 = fv[3 * k + 2];
        fvi[k] = make_int4(i0, i1, i2, 0);
        realize_facet(k, fv, realize_vertex(i0, a, u, r, scale, vcomp, cxf),
                      realize_vertex(i1, a, u, r, scale, vcomp, cxf), realize_vertex(i2, a, u, r, scale, vcomp, cxf),
                      fn, area);
    } else if (k < nf + nv) {
        vx[k - nf] = realize_vertex(k - nf, a, u, r, scale, vcomp, cxf);
    }
}

// vertex normal = normalized sum of attached facet normals, in af order
// (src/shape/realize_mod.c:550-563)
__global__ void k_realize_vnormals(int nv, const int *__restrict__ af_ptr, const int *__restrict__ af_idx,
                                   const double4 *__restrict__ fn, double4 *__restrict__ vn)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    double n0 = 0.0, n1 = 0.0, n2 = 0.0;
    for (int j = af_ptr[i]; j < af_ptr[i + 1]; j++) {
        double4 fnj = fn[af_idx[j]];
        n0 += fnj.x; n1 += fnj.y; n2 += fnj.z;
    }
    double norm = 0.0;
    norm += n0 * n0;
    norm += n1 * n1;
    norm += n2 * n2;
    norm = sqrt(norm);
    if (norm != 0.0) {
        n0 /= norm; n1 /= norm; n2 /= norm;
    }
    vn[i] = make_double4(n0, n1, n2, 0.0);
}

// ------------------------------------------------------------- transforms

__device__ inline void store_vt(double4 *vt, int i, double x, double y, double z)
{
    vt[i] = make_double4(x, y, z, 0.0);
}

// Vertex coordinates in each view's frame: cotrans(v, oa, x, 1) then
// += orbit_offset (src/shape/posvis.c:159-166; 0.0 for the engine's views).
template <typename T4>
__global__ void k_xform(const FrameGeom *__restrict__ geoms, const double4 *__restrict__ vx, int nv,
                        T4 *__restrict__ vt)
{
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const FrameGeom &g = geoms[blockIdx.y];
    double4 x = vx[i];
    double t[3];
#pragma unroll
    for (int r = 0; r < 3; r++) {
        t[r] = 0.0;
        t[r] += g.oa[3 * r + 0] * x.x;
        t[r] += g.oa[3 * r + 1] * x.y;
        t[r] += g.oa[3 * r + 2] * x.z;
        t[r] += g.off[r];
    }
    store_vt(vt, g.vt_base + i, t[0], t[1], t[2]);
}

// The same transform of vertices realized on the fly (realize_vertex, the
// operations k_realize_vf uses), so the batched graph can run it beside
// k_realize_vf instead of after it: the view-frame vertices are identical.
template <typename T4>
__global__ void k_xform_realize(const FrameGeom *__restrict__ geoms, const double *__restrict__ a,
                                const double *__restrict__ u, const double *__restrict__ r,
                                const double *__restrict__ scale, const int *__restrict__ vcomp,
                                const double *__restrict__ cxf, int nv, T4 *__restrict__ vt)
{
    grid_dep_wait();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nv) return;
    const FrameGeom &g = geoms[blockIdx.y];
    double4 x = realize_vertex(i, a, u, r, scale, vcomp, cxf);
    double t[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
        t[k] = 0.0;
        t[k] += g.oa[3 * k + 0] * x.x;
        t[k] += g.oa[3 * k + 1] * x.y;
        t[k] += g.oa[3 * k + 2] * x.z;
        t[k] += g.off[k];
    }
    store_vt(vt, g.vt_base + i, t[0], t[1], t[2]);
}

// -------------------------------------------------------------- binning

// Resident 256-thread blocks per SM the binning kernel's registers must
// allow: it waits on dependent loads (normal and corners, then the bin
// atomics), so more blocks in flight hide more of that latency.
#ifndef BIN_MIN_BLOCKS
#define BIN_MIN_BLOCKS 6
#endif

// Facet culling, bounding box, outbnd flag and POSrect bookkeeping of
// posvis (src/shape/posvis.c:142-199, 322-364), then one bin entry per
// overlapped 16x16 tile. Bin order is arbitrary; the raster kernel sorts.
template <typename T4>
__global__ void __launch_bounds__(256, BIN_MIN_BLOCKS) k_bin(const FrameGeom *__restrict__ geoms, int view0, int nf,
                      const int4 *__restrict__ fvi, const double4 *__restrict__ fn,
                      const T4 *__restrict__ vt, FrameState *__restrict__ states,
                      int *__restrict__ bin_count, int2 *__restrict__ bin_ids, int cap)
{
    grid_dep_wait();
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    int v = view0 + blockIdx.y;
    const FrameGeom &g = geoms[v];
    // the normal and the corner indices load together (the culling test
    // does not wait for the indices); the corners follow
    const double4 nb = fn[f];
    const int4 c = fvi[f];
    double nz = 0.0;
    nz += g.oa[6] * nb.x;
    nz += g.oa[7] * nb.y;
    nz += g.oa[8] * nb.z;
    if (!(nz > 0.0)) return;
    T4 p0 = vt[g.vt_base + c.x], p1 = vt[g.vt_base + c.y], p2 = vt[g.vt_base + c.z];
    const double kmpp = g.kmpp;
    const int n = g.n;
    double xmin = dmin_((double)p0.x, dmin_((double)p1.x, (double)p2.x));
    double xmax = dmax_((double)p0.x, dmax_((double)p1.x, (double)p2.x));
    double ymin = dmin_((double)p0.y, dmin_((double)p1.y, (double)p2.y));
    double ymax = dmax_((double)p0.y, dmax_((double)p1.y, (double)p2.y));
    double imin_d = floor(xmin / kmpp - SMALLVAL + 0.5);
    double imax_d = floor(xmax / kmpp + SMALLVAL + 0.5);
    double jmin_d = floor(ymin / kmpp - SMALLVAL + 0.5);
    double jmax_d = floor(ymax / kmpp + SMALLVAL + 0.5);
    int imin = clamp_lo(imin_d), imax = clamp_hi(imax_d);
    int jmin = clamp_lo(jmin_d), jmax = clamp_hi(jmax_d);
    FrameState &st = states[v];
    if (imin < -n || imax > n || jmin < -n || jmax > n)
        st.outbnd = 1;
    int i1 = max(imin, -n), i2 = min(imax, n), j1 = max(jmin, -n), j2 = min(jmax, n);
    if (i1 > n || i2 < -n || j1 > n || j2 < -n) {
        atomicMin(&st.ofr_i[0], max(imin, -n));
        atomicMax(&st.ofr_i[1], min(imax, n));
        atomicMin(&st.ofr_j[0], max(jmin, -n));
        atomicMax(&st.ofr_j[1], min(jmax, n));
        atomicMin(&st.ofr_ov[0], dkey(imin_d));
        atomicMax(&st.ofr_ov[1], dkey(imax_d));
        atomicMin(&st.ofr_ov[2], dkey(jmin_d));
        atomicMax(&st.ofr_ov[3], dkey(jmax_d));
        return;
    }
    int tx0 = (i1 + n) / TILE_W, tx1 = (i2 + n) / TILE_W;
    int ty0 = (j1 + n) / TILE_W, ty1 = (j2 + n) / TILE_W;
    {
        // facets inside one tile (most of them): lanes of a warp with the
        // same tile reserve their slots with one atomic
        const unsigned act = __activemask();
        const bool single = (tx0 == tx1) && (ty0 == ty1);
        const unsigned sm = __ballot_sync(act, single);
        if (single) {
            const int tile = g.tile_base + tx0 * g.tiles_x + ty0;
            const int lane = threadIdx.x & 31;
            const unsigned peers = __match_any_sync(sm, tile);
            const int leader = __ffs(peers) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(&bin_count[tile], __popc(peers));
            base = __shfl_sync(peers, base, leader);
            const int slot = base + __popc(peers & ((1u << lane) - 1u));
            if (slot < cap) {
                int ti0 = -n + tx0 * TILE_W, tj0 = -n + ty0 * TILE_W;
                int ri1 = max(i1, ti0) - ti0, ri2 = min(i2, ti0 + TILE_W - 1) - ti0;
                int rj1 = max(j1, tj0) - tj0, rj2 = min(j2, tj0 + TILE_W - 1) - tj0;
                bin_ids[(size_t)tile * cap + slot] = make_int2(f, ri1 | (ri2 << 4) | (rj1 << 8) | (rj2 << 12));
            } else {
                st.bin_overflow = 1;
            }
            return;
        }
    }
    for (int tx = tx0; tx <= tx1; tx++)
        for (int ty = ty0; ty <= ty1; ty++) {
            int tile = g.tile_base + tx * g.tiles_x + ty;
            int slot = atomicAdd(&bin_count[tile], 1);
            if (slot < cap) {
                // bbox clipped to the tile, relative to its corner, 4 bits per bound
                int ti0 = -n + tx * TILE_W, tj0 = -n + ty * TILE_W;
                int ri1 = max(i1, ti0) - ti0, ri2 = min(i2, ti0 + TILE_W - 1) - ti0;
                int rj1 = max(j1, tj0) - tj0, rj2 = min(j2, tj0 + TILE_W - 1) - tj0;
                bin_ids[(size_t)tile * cap + slot] = make_int2(f, ri1 | (ri2 << 4) | (rj1 << 8) | (rj2 << 12));
            } else {
                st.bin_overflow = 1;
            }
        }
}

__global__ void k_reset_state(FrameState *st, int nviews, int *bin_count, int ntiles)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nviews) {
        FrameState s;
        s.outbnd = 0;
        s.bin_overflow = 0;
        s.cov_i[0] = s.cov_j[0] = INT_MAX;
        s.cov_i[1] = s.cov_j[1] = INT_MIN;
        s.ofr_i[0] = s.ofr_j[0] = INT_MAX;
        s.ofr_i[1] = s.ofr_j[1] = INT_MIN;
        s.ofr_ov[0] = s.ofr_ov[2] = dkey(HUGENUMBER);
        s.ofr_ov[1] = s.ofr_ov[3] = dkey(-HUGENUMBER);
        s.idellim[0] = s.idoplim[0] = INT_MAX;
        s.idellim[1] = s.idoplim[1] = INT_MIN;
        s.dellim[0] = s.doplim[0] = dkey(HUGENUMBER);
        s.dellim[1] = s.doplim[1] = dkey(-HUGENUMBER);
        s.any_lit = 0;
        s.any_overflow = 0;
        st[i] = s;
    }
    for (int t = i; t < ntiles; t += gridDim.x * blockDim.x)
        bin_count[t] = 0;
}

// ----------------------------------------------------------------- chi2

// Neumaier-compensated accumulator.
struct KSum {
    double s, c;
    __device__ void add(double x)
    {
        double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
    __device__ void merge(const KSum &o)
    {
        add(o.s);
        c += o.c;
    }
    __device__ double value() const { return s + c; }
};

__device__ inline KSum shfl_ksum(KSum a, int off)
{
    KSum b;
    b.s = __shfl_down_sync(0xffffffffu, a.s, off);
    b.c = __shfl_down_sync(0xffffffffu, a.c, off);
    return b;
}

// Per (frame, chunk) partial sums of chi2_deldop (src/shape/chi2.c:436-441):
// o2 = sum obs^2/var, m2 = sum fit^2/var, om = sum fit*obs/var, each
// product in the reference's order, accumulated with compensation.
template <typename T>
__device__ void chi2_item_warp(const Chi2Args &a, int it, const Chi2Item &item, double *part);

// Resident 256-thread blocks per SM of the chi-square kernels: a warp keeps
// its item's 48 loads in flight, so residency trades against registers (on
// 64 uneven frames: 3 blocks, 80 registers, 28.6 us; 2 blocks, 120
// registers, 31.5 us; 4 blocks, 64 registers, 30.7 us).
#ifndef CHI2_MIN_BLOCKS
#define CHI2_MIN_BLOCKS 3
#endif

// One warp per item, items in grid-stride order over the block's warps.
template <typename T>
__global__ void __launch_bounds__(CHI2_THREADS, CHI2_MIN_BLOCKS) k_chi2_partials(Chi2Args a)
{
    const int wpb = blockDim.x >> 5;
    for (int it = blockIdx.x * wpb + (threadIdx.x >> 5); it < a.nitems; it += gridDim.x * wpb)
        chi2_item_warp<T>(a, it, a.items[it], a.partials + (size_t)it * 6);
}

// A frame's three sums from its item partials (6 per item: o2, m2, om, each
// a compensated sum and its compensation) in one fixed order: lane l of a
// warp merges items l, l+32, l+64, ... in turn, then the lanes' sums merge
// pairwise (l with l+16, l+8, ..., l+1), and the frame's start values (a
// Doppler frame's overflow o2 and m2, else 0) take the result last.
// frame_sums_warp does this with the 32 lanes; frame_sums_serial computes
// the same numbers in one thread, so the batched and plain forms agree
// bit for bit.
__device__ inline void ksum_take(KSum &q, const double *p)
{
    q.add(p[0]);
    q.c += p[1];
}
__device__ void frame_sums_warp(const double *part, int nitems, const double start[3], KSum out[3], bool via_l2)
{
    const int lane = threadIdx.x & 31;
    KSum q[3] = {{0, 0}, {0, 0}, {0, 0}};
    for (int it = lane; it < nitems; it += 32)
        for (int k = 0; k < 3; k++) {
            double p[2];
            p[0] = via_l2 ? __ldcg(part + (size_t)it * 6 + 2 * k) : part[(size_t)it * 6 + 2 * k];
            p[1] = via_l2 ? __ldcg(part + (size_t)it * 6 + 2 * k + 1) : part[(size_t)it * 6 + 2 * k + 1];
            ksum_take(q[k], p);
        }
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 3; k++) q[k].merge(shfl_ksum(q[k], off));
    for (int k = 0; k < 3; k++) {
        out[k].s = start[k];
        out[k].c = 0.0;
        out[k].merge(q[k]);
    }
}
__device__ void frame_sums_serial(const double *part, int nitems, const double start[3], KSum out[3])
{
    KSum q[32][3];
    for (int l = 0; l < 32; l++)
        for (int k = 0; k < 3; k++) q[l][k] = KSum{0, 0};
    for (int it = 0; it < nitems; it++)
        for (int k = 0; k < 3; k++) ksum_take(q[it & 31][k], part + (size_t)it * 6 + 2 * k);
    for (int off = 16; off > 0; off >>= 1)
        for (int l = 0; l < off; l++)
            for (int k = 0; k < 3; k++) q[l][k].merge(q[l + off][k]);
    for (int k = 0; k < 3; k++) {
        out[k].s = start[k];
        out[k].c = 0.0;
        out[k].merge(q[0][k]);
    }
}

// A frame's chi-square terms: chi2_deldop's sums, calibration and
// chi-square (src/shape/chi2.c:436-460) from the frame's item partials.
// part: the chi-square partials (6 per item), in global or shared memory;
// part0: the index of the frame's first item in part. One thread.
__device__ inline void frame_start(const FinalizeArgs &a, const FrameHost &h, double start[3])
{
    // a Doppler frame's sums start from its overflow spectrum's o2 and m2
    // (src/shape/chi2.c:745-747)
    const double *ovf = (h.dop_index >= 0) ? a.ovf_out + (size_t)h.dop_index * DOP_OVF_TERMS : nullptr;
    start[0] = ovf ? ovf[0] : 0.0;
    start[1] = ovf ? ovf[1] : 0.0;
    start[2] = 0.0;
}
__device__ void frame_chi2_from_sums(const FrameHost &h, const KSum q[3], shape_deldop_result &r)
{
    double o2 = q[0].value(), m2 = q[1].value(), om = q[2].value();
    double cal = h.cal_in;
    if (h.cal_floating)
        cal = (om > 0.0) ? om / m2 : SHAPE_TINYCALFACT;
    r.o2 = o2; r.m2 = m2; r.om = om; r.cal = cal;
    r.chi2 = h.weight * (o2 - 2 * cal * om + cal * cal * m2);
}
__device__ void finalize_frame_chi2(const FinalizeArgs &a, int fr, const double *part, int part0,
                                    shape_deldop_result &r)
{
    const FrameHost &h = a.fh[fr];
    double start[3];
    frame_start(a, h, start);
    KSum q[3];
    frame_sums_serial(part + (size_t)part0 * 6, h.nitems, start, q);
    frame_chi2_from_sums(h, q, r);
}

// A frame's posvis / pos2deldop outputs (limits, flags, log-factors), which
// do not depend on the chi-square sums.
__device__ void finalize_frame_geom(const FinalizeArgs &a, int fr, shape_deldop_result &r)
{
    const FrameHost &h = a.fh[fr];
    const FrameGeom &g = a.geoms[h.view];
    const FrameState &st = a.states[h.view];
    const double *ovf = (h.dop_index >= 0) ? a.ovf_out + (size_t)h.dop_index * DOP_OVF_TERMS : nullptr;
    const int n = g.n;
    r.xlim[0] = min(n, min(st.cov_i[0], st.ofr_i[0]));
    r.xlim[1] = max(-n, max(st.cov_i[1], st.ofr_i[1]));
    r.ylim[0] = min(n, min(st.cov_j[0], st.ofr_j[0]));
    r.ylim[1] = max(-n, max(st.cov_j[1], st.ofr_j[1]));
    r.outbnd = st.outbnd;
    r.posbnd_logfactor = 0.0;
    if (st.outbnd) {
        double oimin = dkey_inv(st.ofr_ov[0]), oimax = dkey_inv(st.ofr_ov[1]);
        double ojmin = dkey_inv(st.ofr_ov[2]), ojmax = dkey_inv(st.ofr_ov[3]);
        if (st.cov_i[0] != INT_MAX) {
            oimin = dmin_(oimin, (double)st.cov_i[0]);
            oimax = dmax_(oimax, (double)st.cov_i[1]);
            ojmin = dmin_(ojmin, (double)st.cov_j[0]);
            ojmax = dmax_(ojmax, (double)st.cov_j[1]);
        }
        double xfactor = (dmax_(oimax, n) - dmin_(oimin, -n) + 1) / (2 * n + 1);
        double yfactor = (dmax_(ojmax, n) - dmin_(ojmin, -n) + 1) / (2 * n + 1);
        r.posbnd_logfactor = log(xfactor * yfactor);
    }
    r.badradar = h.badradar;
    r.badradar_logfactor = h.badradar_logfactor;
    if (ovf && ovf[4] != 0.0) {       // model wider than the overflow spectrum
        r.badradar = 1;
        r.badradar_logfactor += ovf[5];
    }
    r.idellim[0] = min(g.ndel + 999999, st.idellim[0]);
    r.idellim[1] = max(-999999, st.idellim[1]);
    r.idoplim[0] = min(g.ndop + 999999, st.idoplim[0]);
    r.idoplim[1] = max(-999999, st.idoplim[1]);
    double dl0 = dmin_(HUGENUMBER, dkey_inv(st.dellim[0])), dl1 = dmax_(-HUGENUMBER, dkey_inv(st.dellim[1]));
    double pl0 = dmin_(HUGENUMBER, dkey_inv(st.doplim[0])), pl1 = dmax_(-HUGENUMBER, dkey_inv(st.doplim[1]));
    double dpp = a.set_delpp[h.set], fpp = a.set_doppp[h.set];
    r.dellim[0] = (dl0 - g.delshift) * dpp;
    r.dellim[1] = (dl1 - g.delshift) * dpp;
    r.doplim[0] = (pl0 - g.dopshift) * fpp - a.dop_extra[fr];
    r.doplim[1] = (pl1 - g.dopshift) * fpp + a.dop_extra[fr];
    if (g.dop1d) {                    // a spectrum has no delay axis
        r.idellim[0] = r.idellim[1] = 0;
        r.dellim[0] = r.dellim[1] = 0.0;
    }
}

// Per-frame results: both parts, stored in a.results[fr].
__device__ shape_deldop_result finalize_frame(const FinalizeArgs &a, int fr, const double *part, int part0)
{
    shape_deldop_result r;
    finalize_frame_chi2(a, fr, part, part0, r);
    finalize_frame_geom(a, fr, r);
    a.results[fr] = r;
    return r;
}


// Overflow spectra of the Doppler frames (src/shape/pos2doppler.c:451-499):
// one block per frame sums the bins inside the frame's Doppler limits
// (count of nonzero bins, squares over the noise variance, cross section and
// its mean bin) and flags a model wider than the overflow spectrum.
__global__ void k_doppler_overflow(DopOvfArgs a)
{
    __shared__ double red[4][32];
    const int k = blockIdx.x;
    const int fr = a.frames[k];
    const FrameHost &h = a.fh[fr];
    const FrameGeom &g = a.geoms[h.view];
    const FrameState &st = a.states[h.view];
    double *out = a.out + (size_t)k * DOP_OVF_TERMS;
    if (!st.any_overflow) {
        if (threadIdx.x < DOP_OVF_TERMS) out[threadIdx.x] = 0.0;
        return;
    }
    const double *ov = a.ovf + g.ovf_base;
    const double variance = h.sdev * h.sdev;
    const int idop0 = g.idop0;
    const int j1 = max(st.idoplim[0] + idop0, 0), j2 = min(st.idoplim[1] + idop0, DOP_MAXOVERFLOW - 1);
    double o2 = 0.0, m2 = 0.0, xs = 0.0, dm = 0.0;
    for (int j = j1 + (int)threadIdx.x; j <= j2; j += blockDim.x) {
        const double v = ov[j];
        if (v != 0.0) {
            o2 += 1.0;
            m2 += v * v / variance;
            xs += v;
            dm += (j - idop0) * v;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        o2 += __shfl_down_sync(0xffffffffu, o2, o);
        m2 += __shfl_down_sync(0xffffffffu, m2, o);
        xs += __shfl_down_sync(0xffffffffu, xs, o);
        dm += __shfl_down_sync(0xffffffffu, dm, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { red[0][w] = o2; red[1][w] = m2; red[2][w] = xs; red[3][w] = dm; }
    __syncthreads();
    if (threadIdx.x == 0) {
        o2 = m2 = xs = dm = 0.0;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ww++) {
            o2 += red[0][ww]; m2 += red[1][ww]; xs += red[2][ww]; dm += red[3][ww];
        }
        if (xs != 0.0) dm /= xs;
        out[0] = o2; out[1] = m2; out[2] = xs; out[3] = dm;
        const int lo = st.idoplim[0] + idop0, hi = st.idoplim[1] + idop0;
        if (lo < 0 || hi >= DOP_MAXOVERFLOW) {
            const double dopfactor = (max(hi, DOP_MAXOVERFLOW) - min(lo, 0)) / (1.0 * DOP_MAXOVERFLOW);
            out[4] = 1.0;
            out[5] = log(dopfactor);
        } else {
            out[4] = 0.0;
            out[5] = 0.0;
        }
    }
}

// ------------------------------------------------------------ lightcurves

// posmask (src/shape/posmask.c:58-174) and apply_photo
// (src/shape/apply_photo.c:85-133, 226-248) per POS pixel of one
// lightcurve point; brightness summed per work item (fixed order within a
// block, items summed in order by k_lc_finalize).
template <typename T>
__global__ void k_lc_photo(LcArgs a)
{
    __shared__ double red[32];
    for (int it = blockIdx.x; it < a.nitems; it += gridDim.x) {
        int2 item = a.items[it];
        const LcPointDev &P = a.pts[item.x];
        const FrameGeom &go = a.geoms[P.obs_view];
        const FrameGeom &gs = a.geoms[P.sun_view];
        const int n = go.n, side = go.side;
        const long long npix = (long long)side * side;
        const double *Z = a.z + go.pos_base;
        T *CE = static_cast<T *>(a.cose) + go.pos_base;
        const T *CI = static_cast<const T *>(a.cosi) + go.pos_base;
        const double *ZI = a.zill + gs.pos_base;
        const int *F = a.f + go.pos_base;
        const int *FI = a.fill + gs.pos_base;
        const double bignum = 0.99 * HUGENUMBER;
        // a plane-of-sky frame keeps its brightness image (pos->b of
        // apply_photo, zero where nothing is lit)
        double *Bimg = (a.bimg && P.b_base >= 0) ? a.bimg + P.b_base : nullptr;
        double bsum = 0.0;
        long long pend = (long long)item.y + a.chunk;
        if (pend > npix) pend = npix;
        for (long long p = item.y + threadIdx.x; p < pend; p += blockDim.x) {
            double cose = (double)CE[p];
            if (cose == 0.0) {
                if (Bimg) Bimg[p] = 0.0;
                continue;
            }
            int i = (int)(p / side) - n, j = (int)(p % side) - n;
            double xin[3] = {i * go.kmpp, j * go.kmpp, (double)Z[p]};
            double x[3];
#pragma unroll
            for (int r = 0; r < 3; r++) {
                x[r] = 0.0;
                x[r] += P.so[3 * r + 0] * xin[0];
                x[r] += P.so[3 * r + 1] * xin[1];
                x[r] += P.so[3 * r + 2] * xin[2];
            }
            double i0 = x[0] * P.pixels_per_km, j0 = x[1] * P.pixels_per_km;
            int im = iround_(i0), jm = iround_(j0);
#define ZILL(a_, b_) ((double)ZI[(long long)((a_) + n) * side + ((b_) + n)])
            if (fabs(i0) < n && fabs(j0) < n && ZILL(im, jm) > -bignum &&
                F[p] != FI[(long long)(im + n) * side + (jm + n)]) {
                if (posmask_zill(ZI, n, side, i0, j0, im, jm) - x[2] > P.mask_tol) {
                    cose = 0.0;
                    CE[p] = (T)0;
                }
            }
#undef ZILL
            double cosi = (double)CI[p];
            int f = F[p];
            if (a.mark_seen && cose > a.mincosine_seen && cosi > a.mincosine_seen && f >= 0)
                a.seen[f] = 1;
            double bv = 0.0;
            if (cose > 0.0 && cosi > 0.0 && f >= 0) {
                double b;
                if (P.law_type == SHAPE_OPTLAW_LAMBERT)
                    b = P.intensityfactor * P.scale * cosi;
                else if (P.law_type == SHAPE_OPTLAW_LOMMEL)
                    b = P.intensityfactor * P.scale * cosi / (cosi + cose);
                else
                    b = P.intensityfactor * cosi * (P.s_ls / (cosi + cose) + P.s_l);
                bsum += b;
                bv = b;
            }
            if (Bimg) Bimg[p] = bv;
        }
        for (int off = 16; off > 0; off >>= 1)
            bsum += __shfl_down_sync(0xffffffffu, bsum, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = bsum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
            a.partials[it] = s;
        }
        __syncthreads();
    }
}

// A radar frame's badradar term of the objective (src/shape/calc_fits.c:
// 545-550): dof * log-factor / views, summed over the views whose
// footprint was too wide; the flag when any of them was. One view: the
// frame's own result (which includes a Doppler frame's overflow term).
__device__ inline double frame_blog(const FrameHost &h, double frame_lf)
{
    return h.nviews > 1 ? h.dof * h.badradar_lfsum / h.nviews : h.dof * frame_lf / 1;
}
__device__ inline bool frame_bad(const FrameHost &h, int frame_bad)
{
    return frame_bad || (h.nviews > 1 && h.badradar_any);
}

// posbnd_logfactor of one POS view (src/shape/posvis.c:301-307).
__device__ double view_logfactor(const FrameGeom &g, const FrameState &st)
{
    const int n = g.n;
    double oimin = dkey_inv(st.ofr_ov[0]), oimax = dkey_inv(st.ofr_ov[1]);
    double ojmin = dkey_inv(st.ofr_ov[2]), ojmax = dkey_inv(st.ofr_ov[3]);
    if (st.cov_i[0] != INT_MAX) {
        oimin = dmin_(oimin, (double)st.cov_i[0]);
        oimax = dmax_(oimax, (double)st.cov_i[1]);
        ojmin = dmin_(ojmin, (double)st.cov_j[0]);
        ojmax = dmax_(ojmax, (double)st.cov_j[1]);
    }
    double xfactor = (dmax_(oimax, n) - dmin_(oimin, -n) + 1) / (2 * n + 1);
    double yfactor = (dmax_(ojmax, n) - dmin_(ojmin, -n) + 1) / (2 * n + 1);
    return log(xfactor * yfactor);
}


// ---- plane-of-sky frames (calc_poset, src/shape/calc_fits.c:1156-1330)

// The interpolation polynomial of cubic convolution with parameter -1 (the
// original kernel; resampim's CUBICPAR), in resampim's operations.
__device__ double cubicconv_w(double x)
{
    const double c = -1.0;
    const double ax = fabs(x);
    if (ax < 1) return (c + 2) * ax * ax * ax - (c + 3) * ax * ax + 1;
    if (ax < 2) return c * (ax * ax * ax - 5 * ax * ax + 8 * ax - 4);
    return 0.0;
}

// One sample of the resampling grid (src/util/resampim.c): the grid point
// of temporary column it and row jt, reached by resampim's running sums
// (x1start and y1start advance once per column, x1 and y1 once per row),
// read from the brightness image B ([-n..n]^2, j contiguous) by the
// frame's interpolation; 0 where the input pixels it needs leave the image.
__device__ double poset_sample(const double *B, int n, int side, int mode, double x1start, double y1start,
                               double dxx, double dyx, double dxy, double dyy, int it, int jt)
{
    double x1 = x1start, y1 = y1start;
    for (int k = 1; k < it; k++) { x1 += dxx; y1 += dyx; }
    for (int k = 1; k < jt; k++) { x1 += dxy; y1 += dyy; }
#define IM(i_, j_) B[(long long)((i_) + n) * side + ((j_) + n)]
    if (mode == SHAPE_RESAMPLE_NONE || mode == SHAPE_RESAMPLE_NEAREST) {
        const int ix = iround_(x1), iy = iround_(y1);
        return (ix >= -n && ix <= n && iy >= -n && iy <= n) ? IM(ix, iy) : 0.0;
    }
    const int ix = (int)floor(x1), iy = (int)floor(y1);
    if (mode == SHAPE_RESAMPLE_BILINEAR) {
        if (!(ix >= -n && ix < n && iy >= -n && iy < n)) return 0.0;
        const double t = x1 - ix, u = y1 - iy;
        return (1 - t) * (1 - u) * IM(ix, iy) + t * (1 - u) * IM(ix + 1, iy) + t * u * IM(ix + 1, iy + 1) +
               (1 - t) * u * IM(ix, iy + 1);
    }
    // cubic convolution: four interpolations along rows, then one along the column
    double v = 0.0;
    if (ix > -n && ix < n - 1 && iy > -n && iy < n - 1) {
        const double t = x1 - ix, u = y1 - iy;
        double xp[4];
        for (int k = -1; k <= 2; k++) xp[k + 1] = cubicconv_w(k - t);
        for (int l = -1; l <= 2; l++) {
            double xi = 0.0;
            for (int k = -1; k <= 2; k++) xi += xp[k + 1] * IM(ix + k, iy + l);
            v += cubicconv_w(l - u) * xi;
        }
    }
    return v;
#undef IM
}

// One block per plane-of-sky frame: the fit image by resampim (with
// rebinning when the grid undersamples the rendering by an integer factor
// and image_rebin is set; cubic convolution clipped at 0), checkposet's
// test of the lit pixels' corners against the rotated fit grid
// (src/util/checkposet.c), chi2_poset's sums with the floating
// calibration (src/shape/chi2.c) and the views' posbnd terms.
__global__ void k_poset_frames(PosetArgs a)
{
    __shared__ double red[5][32];
    __shared__ int redi[32];
    const PosetFrameDev F = a.frames[blockIdx.x];
    const LcPointDev &P = a.pts[F.point];
    const FrameGeom &go = a.geoms[P.obs_view], &gs = a.geoms[P.sun_view];
    const int n = go.n, side = go.side;
    const double *B = a.bimg + P.b_base;
    const int ncol = F.ncol, nrow = F.nrow;
    double *FIT = a.fit + F.img_base;
    const double *OBS = a.obs + F.img_base, *OOV = a.oov + F.img_base;
    // resampim's grid over the temporary image (1..xt2) x (1..yt2)
    int xb = 1, yb = 1;
    if (F.rebin) {
        xb = max(iround_(F.xwidth / (ncol - 1)), 1);
        yb = max(iround_(F.ywidth / (nrow - 1)), 1);
    }
    const int npix = xb * yb;
    const bool rebin = F.rebin && npix > 1;
    const int xt2 = rebin ? xb * ncol : ncol, yt2 = rebin ? yb * nrow : nrow;
    const double xstep = (F.mode == SHAPE_RESAMPLE_NONE) ? 1.0 : F.xwidth / (xt2 - 1);
    const double ystep = (F.mode == SHAPE_RESAMPLE_NONE) ? 1.0 : F.ywidth / (yt2 - 1);
    const double dxx = xstep * F.cosang, dxy = ystep * F.sinang;
    const double dyx = -xstep * F.sinang, dyy = ystep * F.cosang;
    const double x1s = F.x0 - ((xt2 - 1) / 2.0) * dxx - ((yt2 - 1) / 2.0) * dxy;
    const double y1s = F.y0 - ((xt2 - 1) / 2.0) * dyx - ((yt2 - 1) / 2.0) * dyy;
    double o2 = 0.0, m2 = 0.0, om = 0.0;
    for (int p = threadIdx.x; p < ncol * nrow; p += blockDim.x) {
        const int i = p / nrow + 1, j = p % nrow + 1;
        double v;
        if (rebin) {
            v = 0.0;
            for (int k = 1 + (i - 1) * xb; k < 1 + i * xb; k++)
                for (int l = 1 + (j - 1) * yb; l < 1 + j * yb; l++)
                    v += poset_sample(B, n, side, F.mode, x1s, y1s, dxx, dyx, dxy, dyy, k, l);
            v /= npix;
        } else {
            v = poset_sample(B, n, side, F.mode, x1s, y1s, dxx, dyx, dxy, dyy, i, j);
        }
        if (F.mode == SHAPE_RESAMPLE_CUBICCONV) v = fmax(0.0, v);
        FIT[p] = v;
        const double ob = OBS[p], w = OOV[p];
        o2 += ob * ob * w;
        m2 += v * v * w;
        om += v * ob * w;
    }
    // checkposet: every corner of a lit POS pixel against the fit grid
    const double xl1 = -F.xwidth / 2 - 0.5, xl2 = F.xwidth / 2 + 0.5;
    const double yl1 = -F.ywidth / 2 - 0.5, yl2 = F.ywidth / 2 + 0.5;
    double xmin = xl1, xmax = xl2, ymin = yl1, ymax = yl2;
    int bad = 0;
    const int cside = side + 1;
    for (int c = threadIdx.x; c < cside * cside; c += blockDim.x) {
        const int ci = c / cside - n, cj = c % cside - n;      // corner (ci, cj): ci, cj = -n..n+1
        bool lit = false;
        for (int di = -1; di <= 0 && !lit; di++)
            for (int dj = -1; dj <= 0 && !lit; dj++) {
                const int pi = ci + di, pj = cj + dj;
                if (pi >= -n && pi <= n && pj >= -n && pj <= n && B[(long long)(pi + n) * side + (pj + n)] > 0.0)
                    lit = true;
            }
        if (!lit) continue;
        const double xs = (ci - 0.5) - F.x0, ys = (cj - 0.5) - F.y0;
        const double xf = xs * F.cosang + ys * F.sinang;
        const double yf = -xs * F.sinang + ys * F.cosang;
        if (xf < xl1) { bad = 1; xmin = fmin(xmin, xf); }
        else if (xf > xl2) { bad = 1; xmax = fmax(xmax, xf); }
        if (yf < yl1) { bad = 1; ymin = fmin(ymin, yf); }
        else if (yf > yl2) { bad = 1; ymax = fmax(ymax, yf); }
    }
    // block reductions: sums, extremes, the flag
    for (int off = 16; off > 0; off >>= 1) {
        o2 += __shfl_down_sync(0xffffffffu, o2, off);
        m2 += __shfl_down_sync(0xffffffffu, m2, off);
        om += __shfl_down_sync(0xffffffffu, om, off);
        xmin = fmin(xmin, __shfl_down_sync(0xffffffffu, xmin, off));
        xmax = fmax(xmax, __shfl_down_sync(0xffffffffu, xmax, off));
        ymin = fmin(ymin, __shfl_down_sync(0xffffffffu, ymin, off));
        ymax = fmax(ymax, __shfl_down_sync(0xffffffffu, ymax, off));
        bad |= __shfl_down_sync(0xffffffffu, bad, off);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    __shared__ double ext[4][32];
    if (lane == 0) {
        red[0][wid] = o2; red[1][wid] = m2; red[2][wid] = om;
        ext[0][wid] = xmin; ext[1][wid] = xmax; ext[2][wid] = ymin; ext[3][wid] = ymax;
        redi[wid] = bad;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    o2 = m2 = om = 0.0;
    for (int w = 0; w < nw; w++) {
        o2 += red[0][w]; m2 += red[1][w]; om += red[2][w];
        xmin = fmin(xmin, ext[0][w]); xmax = fmax(xmax, ext[1][w]);
        ymin = fmin(ymin, ext[2][w]); ymax = fmax(ymax, ext[3][w]);
        bad |= redi[w];
    }
    shape_poset_result r;
    r.o2 = o2; r.m2 = m2; r.om = om;
    r.cal = (om > 0.0) ? om / m2 : SHAPE_TINYCALFACT;
    r.chi2 = F.weight * (o2 - 2 * r.cal * om + r.cal * r.cal * m2);
    r.badposet = bad;
    r.badposet_logfactor = bad ? log((xmax - xmin) * (ymax - ymin) / ((F.xwidth + 1) * (F.ywidth + 1))) : 0.0;
    const FrameState &so = a.states[P.obs_view], &ss = a.states[P.sun_view];
    r.outbnd = (so.outbnd ? 1 : 0) | (ss.outbnd ? 2 : 0);
    r.posbnd_logsum = 0.0;
    if (so.outbnd) r.posbnd_logsum += 0.5 * F.dof * view_logfactor(go, so);
    if (ss.outbnd) r.posbnd_logsum += 0.5 * F.dof * view_logfactor(gs, ss);
    a.res[blockIdx.x] = r;
}

// Natural cubic spline second derivatives and evaluation (the role of
// spline/splint in src/shape/calc_fits.c:1923-1933). The tridiagonal system
//   h[i-1] y2[i-1] + 2 (h[i-1] + h[i]) y2[i] + h[i] y2[i+1]
//     = 6 ((y[i+1]-y[i])/h[i] - (y[i]-y[i-1])/h[i-1]),   y2[0] = y2[n-1] = 0,
// is solved with each row divided by its span x[i+1] - x[i-1] (lower
// coefficient w = h[i-1]/span, diagonal 2, upper 1 - w): forward
// elimination keeps each row's multiplier of y2[i+1] in y2[i] and its
// eliminated right-hand side in r[i], back substitution forms
// y2[i] = y2[i] y2[i+1] + r[i]. The reference solves the span-scaled rows in
// this order, so the FP64 fits are bit-identical to its.
__device__ void spline_natural_dev(const double *x, const double *y, int n, double *y2, double *r)
{
    if (n < 1) return;
    y2[0] = r[0] = 0.0;
    for (int i = 1; i < n - 1; i++) {
        const double span = x[i + 1] - x[i - 1];
        const double w = (x[i] - x[i - 1]) / span;
        const double piv = w * y2[i - 1] + 2.0;
        y2[i] = (w - 1.0) / piv;
        const double dslope = (y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
        r[i] = (6.0 * dslope / span - w * r[i - 1]) / piv;
    }
    if (n > 1) y2[n - 1] = 0.0;
    for (int i = n - 2; i >= 0; i--) y2[i] = y2[i] * y2[i + 1] + r[i];
}

__device__ double splint_dev(const double *x, const double *y, const double *y2, int n, double t)
{
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (x[mid] > t) hi = mid; else lo = mid;
    }
    double h = x[hi] - x[lo];
    double wl = (x[hi] - t) / h, wh = (t - x[lo]) / h;
    return wl * y[lo] + wh * y[hi] +
           ((wl * wl * wl - wl) * y2[lo] + (wh * wh * wh - wh) * y2[hi]) * (h * h) / 6.0;
}

// One block per lightcurve set: y from brightness partials, spline to the
// observation epochs, chi2_lghtcrv (src/shape/chi2.c:1125-1170), posbnd sum
// (src/shape/calc_fits.c:1651-1679, 1947).
//
// The recurrences (spline elimination, the chi-square sums, the log-factor
// sum) stay serial in the reference's order, so results are bit-identical to
// it; when a.smem_per_set > 0 their operands are first gathered into shared
// memory by the whole block, so the serial loops run at shared-memory latency
// instead of one global round trip per step.
__global__ void k_lc_finalize(LcFinalizeArgs a)
{
    extern __shared__ double lsm[];
    const LcSetDev &S = a.sets[blockIdx.x];
    const int np = S.npts, n = S.n;
    const bool use_sm = a.smem_per_set > 0;
    // shared layout: x y y2 cp [np] | t obs oov fit [n] | lo ls [np] (doubles), flags [np] (int)
    double *x = use_sm ? lsm : const_cast<double *>(S.x);
    double *y = use_sm ? lsm + np : S.y;
    double *y2 = use_sm ? lsm + 2 * np : S.y2;
    double *cp = use_sm ? lsm + 3 * np : S.fit + n;       // global path: fit tail is scratch
    double *tt = use_sm ? lsm + 4 * np : const_cast<double *>(S.t);
    double *obs = use_sm ? tt + n : const_cast<double *>(S.obs);
    double *oov = use_sm ? tt + 2 * n : const_cast<double *>(S.oov);
    double *fit = use_sm ? tt + 3 * n : S.fit;
    double *lo = tt + 4 * n, *ls = lo + np;
    int *pflag = reinterpret_cast<int *>(ls + np);
    for (int k = threadIdx.x; k < np; k += blockDim.x) {
        int pt = S.pt0 + k;
        int it0 = a.pt_items[2 * pt], cnt = a.pt_items[2 * pt + 1];
        double sum = 0.0;
        for (int it = it0; it < it0 + cnt; it++) sum += a.partials[it];
        sum = (sum == 0.0) ? 1.0e-40 : sum;
        y[k] = sum;
        if (use_sm) {
            S.y[k] = sum;
            x[k] = S.x[k];
            // per-point posbnd log-factor terms, summed serially below
            const LcPointDev &P = a.pts[pt];
            const FrameState &so = a.states[P.obs_view], &ss = a.states[P.sun_view];
            lo[k] = so.outbnd ? 0.5 * view_logfactor(a.geoms[P.obs_view], so) : 0.0;
            ls[k] = ss.outbnd ? 0.5 * view_logfactor(a.geoms[P.sun_view], ss) : 0.0;
            pflag[k] = (so.outbnd ? 1 : 0) | (ss.outbnd ? 2 : 0);
        }
    }
    if (use_sm)
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            tt[k] = S.t[k];
            obs[k] = S.obs[k];
            oov[k] = S.oov[k];
        }
    __syncthreads();
    if (threadIdx.x == 0) spline_natural_dev(x, y, np, y2, cp);
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        double v = splint_dev(x, y, y2, np, tt[k]) / 1;
        fit[k] = v;
        if (use_sm) S.fit[k] = v;
    }
    if (use_sm)
        for (int k = threadIdx.x; k < np; k += blockDim.x) S.y2[k] = y2[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        double o2 = 0.0, m2 = 0.0, om = 0.0;
        for (int k = 0; k < n; k++) {
            o2 += obs[k] * obs[k] * oov[k];
            m2 += fit[k] * fit[k] * oov[k];
            om += fit[k] * obs[k] * oov[k];
        }
        double cal = S.cal_in;
        if (S.cal_floating)
            cal = (om > 0.0) ? om / m2 : SHAPE_TINYCALFACT;
        double chi2 = S.weight * (o2 - 2 * cal * om + cal * cal * m2);
        int posbnd = 0;
        double lsum = 0.0;
        for (int k = 0; k < np; k++) {
            if (use_sm) {
                if (pflag[k] & 1) { posbnd = 1; lsum += lo[k]; }
                if (pflag[k] & 2) { posbnd = 1; lsum += ls[k]; }
            } else {
                const LcPointDev &P = a.pts[S.pt0 + k];
                const FrameState &so = a.states[P.obs_view], &ss = a.states[P.sun_view];
                if (so.outbnd) { posbnd = 1; lsum += 0.5 * view_logfactor(a.geoms[P.obs_view], so); }
                if (ss.outbnd) { posbnd = 1; lsum += 0.5 * view_logfactor(a.geoms[P.sun_view], ss); }
            }
        }
        double *o = a.set_out + 4 * blockIdx.x;
        o[0] = cal; o[1] = chi2; o[2] = posbnd; o[3] = lsum;
    }
}

// Totals over all sets in dataset order: chi2 (src/shape/chi2.c:270-300),
// the posbnd / badradar flags and log-factors of calc_fits
// (src/shape/calc_fits.c:407-409, 511-550, 1947) and the objective's
// bad-model multipliers (src/shape/bestfit.c:806-866), no penalties.
//
// The totals are serial sums in dataset order (the reference's order). With
// a.smem_frames set, each frame's thread leaves its chi2 and dof-weighted
// log-factor terms in shared memory, so the serial pass reads shared memory
// instead of waiting on one global load per frame.
template <typename Term>
__device__ void summary_totals(const SummaryArgs &a, Term term);

__global__ void k_summary(FinalizeArgs fa, SummaryArgs a)
{
    extern __shared__ double ssm[];
    const bool use_sm = a.smem_frames;
    double *s_chi2 = ssm, *s_plog = ssm + fa.nframes, *s_blog = ssm + 2 * (size_t)fa.nframes;
    unsigned char *s_flag = reinterpret_cast<unsigned char *>(ssm + 3 * (size_t)fa.nframes);
    // the chi-square partials are copied to shared memory by the whole block
    // first, so each frame's serial merge reads shared memory
    const double *part = fa.partials;
    if (use_sm && a.smem_partials) {
        // partials start at the first 16-byte boundary after the flags
        const size_t poff = (25 * (size_t)fa.nframes + 15) & ~(size_t)15;
        double *sp = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(ssm) + poff);
        // 16-byte loads, eight in flight per thread before their stores
        const double2 *src = reinterpret_cast<const double2 *>(fa.partials);
        double2 *dst = reinterpret_cast<double2 *>(sp);
        const int n2 = 3 * a.nitems;
#pragma unroll 8
        for (int k = threadIdx.x; k < n2; k += blockDim.x) dst[k] = src[k];
        __syncthreads();
        part = sp;
    }
    // per-frame results (one thread per frame), then the totals
    for (int fr = threadIdx.x; fr < fa.nframes; fr += blockDim.x) {
        const shape_deldop_result r = finalize_frame(fa, fr, part, fa.fh[fr].item0);
        if (use_sm) {
            s_chi2[fr] = r.chi2;
            s_plog[fr] = a.fh[fr].dof * r.posbnd_logfactor;
            s_blog[fr] = frame_blog(a.fh[fr], r.badradar_logfactor);
            s_flag[fr] = (r.outbnd ? 1 : 0) | (frame_bad(a.fh[fr], r.badradar) ? 2 : 0);
        }
    }
    __syncthreads();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (use_sm)
        summary_totals(a, [&](int f, double &c, double &pl, double &bl, int &fl) {
            c = s_chi2[f]; pl = s_plog[f]; bl = s_blog[f]; fl = s_flag[f];
        });
    else
        summary_totals(a, [&](int f, double &c, double &pl, double &bl, int &fl) {
            const shape_deldop_result &r = a.results[f];
            c = r.chi2;
            pl = a.fh[f].dof * r.posbnd_logfactor;
            bl = frame_blog(a.fh[f], r.badradar_logfactor);
            fl = (r.outbnd ? 1 : 0) | (frame_bad(a.fh[f], r.badradar) ? 2 : 0);
        });
}

// The totals: serial sums over the sets in dataset order (the reference's
// order, src/shape/chi2.c:270-300 and calc_fits.c:407-409), the flags and
// the objective. term(f, chi2, dof*posbnd_logfactor, dof*badradar_logfactor,
// flags) gives radar frame f's terms (flags: 1 outbnd, 2 badradar).
template <typename Term>
__device__ void summary_totals(const SummaryArgs &a, Term term)
{
    double chi2 = 0.0, chi2_dd = 0.0, chi2_lc = 0.0, chi2_ps = 0.0, plog = 0.0, blog = 0.0, pslog = 0.0;
    int posbnd = 0, badradar = 0, badposet = 0;
    for (int s = 0; s < a.nsets; s++) {
        const SetRec &R = a.sets[s];
        double cs = 0.0;
        if (R.type == 2) {
            // plane-of-sky frames: chi2_poset's frame sum; calc_poset's
            // posbnd terms (dof/2 per view) and badposet terms (dof times
            // checkposet's log factor)
            for (int f = R.first; f < R.first + R.count; f++) {
                const shape_poset_result &r = a.ps_res[f];
                cs += r.chi2;
                if (r.outbnd) { posbnd = 1; plog += r.posbnd_logsum; }
                if (r.badposet) { badposet = 1; pslog += a.ps_frames[f].dof * r.badposet_logfactor; }
            }
            chi2_ps += cs;
        } else if (R.type == 0) {
            for (int f = R.first; f < R.first + R.count; f++) {
                double c, pl, bl;
                int fl;
                term(f, c, pl, bl, fl);
                cs += c;
                if (fl & 1) { posbnd = 1; plog += pl; }
                if (fl & 2) { badradar = 1; blog += bl; }
            }
            chi2_dd += cs;
        } else {
            const double *o = a.lc_out + 4 * R.first;
            cs = o[1];
            if (o[2] != 0.0) posbnd = 1;
            plog += a.lc_dof[R.first] * (o[3] / a.lc_npts[R.first]);
            chi2_lc += cs;
        }
        chi2 += cs;
    }
    shape_eval_summary out;
    out.chi2 = chi2;
    out.dof = a.dof;
    out.chi2_deldop = chi2_dd;
    out.chi2_lghtcrv = chi2_lc;
    out.posbnd = posbnd;
    out.posbnd_logfactor = plog / a.dof;
    out.badradar = badradar;
    out.badradar_logfactor = blog / a.dof_radar;
    out.chi2_poset = chi2_ps;
    out.badposet = badposet;
    out.badposet_logfactor = badposet ? pslog / a.dof_poset : 0.0;
    double err = chi2 / a.dof;
    if (a.baddiam) err *= a.bad_objfactor * exp(a.baddiam_logfactor);
    if (posbnd) err *= a.bad_objfactor * exp(out.posbnd_logfactor);
    if (badposet) err *= a.bad_objfactor * exp(out.badposet_logfactor);
    if (badradar) err *= a.bad_objfactor * exp(out.badradar_logfactor);
    out.objective = err;
    out.penalties = 0.0;
    *a.out = out;
}

// One item's chi-square partial sums, left by lane 0 of the calling warp in
// part[0..5]: each lane sums its 16 bins (lane, lane + 32, ...) in order in
// plain FP64, then the lanes' sums merge with compensation by warp shuffles
// (pairwise: l with l+16, l+8, ..., l+1). With a.o2pre set, o2 is the item's
// precomputed partial and obs / 1/var are read only where the fit is
// nonzero: a zero fit bin adds exact zeros to m2 and om, so the sums keep
// their values.
template <typename T>
__device__ void chi2_item_warp(const Chi2Args &a, int it, const Chi2Item &item, double *part)
{
    const int lane = threadIdx.x & 31;
    const FrameGeom &g = a.geoms[a.frame_view[item.frame]];
    const long long base = g.fit_base + item.start;
    const T *fit = static_cast<const T *>(a.fit) + base;
    const double *obs = a.obs + base, *oov = a.oov + base;
    const bool pre = a.o2pre != nullptr;
    T ft[CHI2_LANE];
#pragma unroll
    for (int j = 0; j < CHI2_LANE; j++) {
        const int k = lane + 32 * j;
        ft[j] = (k < item.count) ? fit[k] : (T)0;
    }
    double ob[CHI2_LANE], wv[CHI2_LANE];
#pragma unroll
    for (int j = 0; j < CHI2_LANE; j++) {
        const int k = lane + 32 * j;
        const bool in = (k < item.count) && (!pre || ft[j] != (T)0);
        ob[j] = in ? obs[k] : 0.0;
        wv[j] = in ? oov[k] : 0.0;
    }
    double so2 = 0.0, sm2 = 0.0, som = 0.0;
#pragma unroll
    for (int j = 0; j < CHI2_LANE; j++) {
        if (lane + 32 * j >= item.count) break;
        const double f = (double)ft[j];
        if (!pre) so2 += ob[j] * ob[j] * wv[j];
        sm2 += f * f * wv[j];
        som += f * ob[j] * wv[j];
    }
    KSum o2 = {so2, 0}, m2 = {sm2, 0}, om = {som, 0};
    for (int off = 16; off > 0; off >>= 1) {
        o2.merge(shfl_ksum(o2, off));
        m2.merge(shfl_ksum(m2, off));
        om.merge(shfl_ksum(om, off));
    }
    if (lane == 0) {
        if (pre) {
            o2.s = a.o2pre[2 * (size_t)it];
            o2.c = a.o2pre[2 * (size_t)it + 1];
        }
        part[0] = o2.s; part[1] = o2.c;
        part[2] = m2.s; part[3] = m2.c;
        part[4] = om.s; part[5] = om.c;
    }
}

// Chi-square partials, per-frame results and totals in one launch, warp by
// warp with no block barrier: each warp takes (frame, 512-bin) items in
// grid-stride order. A frame's counter takes one count per item; the warp
// that makes the frame's last count merges the frame's item partials
// (frame_sums_warp, the order k_summary's frame_sums_serial reproduces) and
// writes the frame's results (limits, flags, log-factors and chi-square
// terms), and the warp that completes the last frame computes the totals in
// dataset order, as k_chi2_partials + k_summary do. Values another warp
// wrote in this launch are read through L2 (__ldcg) after a fence.
// counters: [nframes] per frame, then the finished frames; zero before the
// launch.
template <typename T>
__global__ void __launch_bounds__(CHI2_THREADS, CHI2_MIN_BLOCKS) k_chi2_summary(Chi2Args ca, FinalizeArgs fa, SummaryArgs sa,
                                                               int *counters)
{
    extern __shared__ __align__(16) unsigned char stage[];   // chi2_summary_smem bytes (the totals)
    grid_dep_wait();
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int it = blockIdx.x * wpb + (threadIdx.x >> 5); it < ca.nitems; it += gridDim.x * wpb) {
        const Chi2Item item = ca.items[it];
        chi2_item_warp<T>(ca, it, item, ca.partials + (size_t)it * 6);
        const int fr = item.frame;
        const FrameHost &h = fa.fh[fr];
        int last = 0;
        if (lane == 0) {
            __threadfence();                                  // the partials before the count
            last = (atomicAdd(&counters[fr], 1) == h.nitems - 1);
        }
        last = __shfl_sync(full, last, 0);
        if (!last) continue;                                  // warp-uniform
        __threadfence();
        double start[3];
        frame_start(fa, h, start);
        KSum q[3];
        frame_sums_warp(ca.partials + (size_t)h.item0 * 6, h.nitems, start, q, true);
        int lastf = 0;
        if (lane == 0) {
            shape_deldop_result r;
            finalize_frame_geom(fa, fr, r);
            frame_chi2_from_sums(h, q, r);
            fa.results[fr] = r;
            __threadfence();                                  // the results before the count
            lastf = (atomicAdd(&counters[fa.nframes], 1) == fa.nframes - 1);
        }
        lastf = __shfl_sync(full, lastf, 0);
        if (!lastf) continue;
        // the totals: this warp stages every frame's terms in shared memory
        // (the only warp of the grid that uses it), then lane 0 sums them in
        // dataset order
        __threadfence();
        double *s_chi2 = reinterpret_cast<double *>(stage);
        double *s_plog = s_chi2 + fa.nframes, *s_blog = s_plog + fa.nframes;
        unsigned char *s_flag = reinterpret_cast<unsigned char *>(s_blog + fa.nframes);
        for (int f = lane; f < fa.nframes; f += 32) {
            const shape_deldop_result *r = fa.results + f;
            s_chi2[f] = __ldcg(&r->chi2);
            s_plog[f] = fa.fh[f].dof * __ldcg(&r->posbnd_logfactor);
            s_blog[f] = frame_blog(fa.fh[f], __ldcg(&r->badradar_logfactor));
            s_flag[f] = (__ldcg(&r->outbnd) ? 1 : 0) | (frame_bad(fa.fh[f], __ldcg(&r->badradar)) ? 2 : 0);
        }
        __syncwarp();
        if (lane == 0)
            summary_totals(sa, [&](int f, double &c, double &pl, double &bl, int &fl) {
                c = s_chi2[f]; pl = s_plog[f]; bl = s_blog[f]; fl = s_flag[f];
            });
    }
}

}  // namespace

// ------------------------------------------------------------- launchers

void launch_realize_vf(const ModelDev &m, cudaStream_t s)
{
    const int B = 256;
    k_realize_vf<<<(m.nf + m.nv + B - 1) / B, B, 0, s>>>(m.nv, m.nf, m.a, m.u, m.r, m.scale, m.vcomp, m.cxf, m.fv,
                                                          m.vx, m.fn, m.area, m.fvi);
}

void launch_realize_vn(const ModelDev &m, cudaStream_t s)
{
    const int B = 256;
    k_realize_vnormals<<<(m.nv + B - 1) / B, B, 0, s>>>(m.nv, m.af_ptr, m.af_idx, m.fn, m.vn);
}

void launch_realize(const ModelDev &m, cudaStream_t s)
{
    launch_realize_vf(m, s);
    launch_realize_vn(m, s);
}

void launch_reset_state(FrameState *st, int nviews, int *bin_count, int ntiles, cudaStream_t s)
{
    int n = nviews > ntiles ? nviews : ntiles;
    int blocks = (n + 255) / 256;
    if (blocks > 4 * 148) blocks = 4 * 148;
    if (blocks < (nviews + 255) / 256) blocks = (nviews + 255) / 256;
    k_reset_state<<<blocks, 256, 0, s>>>(st, nviews, bin_count, ntiles);
}

void launch_xform_realize_f64(const FrameGeom *g, int nviews, const ModelDev &m, double4 *vt, cudaStream_t s)
{
    dim3 grid((m.nv + 255) / 256, nviews);
    k_xform_realize<double4><<<grid, 256, 0, s>>>(g, m.a, m.u, m.r, m.scale, m.vcomp, m.cxf, m.nv, vt);
}

void launch_xform_f64(const FrameGeom *g, int nviews, const double4 *vx, int nv, double4 *vt, cudaStream_t s,
                      bool pdl)
{
    dim3 grid((nv + 255) / 256, nviews);
    launch_k(k_xform<double4>, grid, dim3(256), 0, s, pdl, g, vx, nv, vt);
}


void launch_bin_f64(const FrameGeom *g, int view0, int nviews, const ModelDev &m, const double4 *vt,
                    FrameState *st, int *bin_count, int2 *bin_ids, int cap, cudaStream_t s, bool pdl)
{
    dim3 grid((m.nf + 255) / 256, nviews);
    launch_k(k_bin<double4>, grid, dim3(256), 0, s, pdl, g, view0, m.nf, (const int4 *)m.fvi, (const double4 *)m.fn,
             vt, st, bin_count, bin_ids, cap);
}


void launch_chi2_partials(const Chi2Args &a, int fp32, cudaStream_t s)
{
    const int wpb = CHI2_THREADS / 32;               // one warp per item
    const int need = (a.nitems + wpb - 1) / wpb;
    int blocks = need < 8 * 148 ? need : 8 * 148;
    if (blocks <= 0) return;
    if (fp32) k_chi2_partials<float><<<blocks, CHI2_THREADS, 0, s>>>(a);
    else k_chi2_partials<double><<<blocks, CHI2_THREADS, 0, s>>>(a);
}

// FP32 form: each Doppler frame's FP64 sums rounded once into its float
// fit bins.
__global__ void k_dop_fit_f32(const int *dop_frames, const FrameHost *fh, const FrameGeom *geoms,
                              const double *fit64, float *fit32)
{
    const FrameGeom &g = geoms[fh[dop_frames[blockIdx.x]].view];
    const long long n = (long long)g.ndel * g.ndop;
    for (long long j = threadIdx.x; j < n; j += blockDim.x) fit32[g.fit_base + j] = (float)fit64[g.fit_base + j];
}

void launch_dop_fit_f32(const int *dop_frames, int n, const FrameHost *fh, const FrameGeom *geoms,
                        const double *fit64, float *fit32, cudaStream_t s)
{
    if (n <= 0) return;
    k_dop_fit_f32<<<n, 256, 0, s>>>(dop_frames, fh, geoms, fit64, fit32);
}

void launch_doppler_overflow(const DopOvfArgs &a, cudaStream_t s)
{
    if (a.n <= 0) return;
    k_doppler_overflow<<<a.n, 256, 0, s>>>(a);
}


void launch_poset_frames(const PosetArgs &a, cudaStream_t s)
{
    if (a.nframes <= 0) return;
    k_poset_frames<<<a.nframes, 256, 0, s>>>(a);
}

void launch_lc_photo(const LcArgs &a, int fp32, cudaStream_t s)
{
    int blocks = a.nitems < 8 * 148 ? a.nitems : 8 * 148;
    if (blocks <= 0) return;
    if (fp32) k_lc_photo<float><<<blocks, 256, 0, s>>>(a);
    else k_lc_photo<double><<<blocks, 256, 0, s>>>(a);
}

// Shared memory one set needs (0 when it exceeds the block's budget: the
// kernel then works on the global arrays).
size_t lc_finalize_smem(int npts, int n)
{
    size_t b = sizeof(double) * (6 * (size_t)npts + 4 * (size_t)n) + sizeof(int) * (size_t)npts;
    return b <= LC_FINALIZE_SMEM_MAX ? b : 0;
}

cudaError_t configure_lc_finalize()
{
    return cudaFuncSetAttribute(k_lc_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)LC_FINALIZE_SMEM_MAX);
}

void launch_lc_finalize(const LcFinalizeArgs &a, cudaStream_t s)
{
    if (a.nsets <= 0) return;
    k_lc_finalize<<<a.nsets, 256, a.smem_per_set, s>>>(a);
}

// Shared memory of the summary: per-frame terms, then (when they fit) the
// chi-square partials; *with_partials tells which.
size_t summary_smem(int nframes, int nitems, int *with_partials)
{
    size_t b = 3 * sizeof(double) * (size_t)nframes + (size_t)nframes;   // terms and flags
    size_t bp = ((b + 15) & ~(size_t)15) + 6 * sizeof(double) * (size_t)nitems;
    *with_partials = bp <= SUMMARY_SMEM_MAX;
    if (*with_partials) return bp;
    return b <= SUMMARY_SMEM_MAX ? b : 0;
}

cudaError_t configure_summary()
{
    return cudaFuncSetAttribute(k_summary, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SUMMARY_SMEM_MAX);
}

size_t chi2_summary_smem(int nframes, int max_frame_items)
{
    (void)max_frame_items;          // a frame's partials merge in registers
    return ((size_t)nframes * 25 + 15) & ~(size_t)15;
}

bool chi2_summary_fits(int nframes, int max_frame_items)
{
    return nframes > 0 && chi2_summary_smem(nframes, max_frame_items) <= FUSED_STAGE_BYTES;
}

void launch_chi2_summary(const Chi2Args &ca, const FinalizeArgs &fa, const SummaryArgs &sa, int *counters,
                         int fp32, cudaStream_t s, bool pdl, size_t smem)
{
    const int wpb = CHI2_THREADS / 32;               // one warp per item
    const int need = (ca.nitems + wpb - 1) / wpb;
    const int blocks = need < 8 * 148 ? need : 8 * 148;
    if (blocks <= 0 || ca.nitems <= 0) return;
    if (fp32) launch_k(k_chi2_summary<float>, dim3(blocks), dim3(CHI2_THREADS), smem, s, pdl, ca, fa, sa, counters);
    else launch_k(k_chi2_summary<double>, dim3(blocks), dim3(CHI2_THREADS), smem, s, pdl, ca, fa, sa, counters);
}

void launch_summary(const FinalizeArgs &fa, const SummaryArgs &a, cudaStream_t s)
{
    SummaryArgs b = a;
    int wp = 0;
    const size_t sm = summary_smem(fa.nframes, a.nitems, &wp);
    b.smem_frames = (sm > 0 && fa.nframes > 0) ? 1 : 0;
    b.smem_partials = b.smem_frames && wp;
    k_summary<<<1, 256, b.smem_frames ? sm : 0, s>>>(fa, b);
}


}  // namespace shape
