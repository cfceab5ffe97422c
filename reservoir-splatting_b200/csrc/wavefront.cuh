// Wavefront form of the ScatterBackup temporal resampling
// (ScatterBackupTemporalResampling.rt.slang:69-283) and of spatial resampling
// (SpatialResampling.rt.slang:67-185).
//
// The shift mappings draw only from a by-value copy of the pixel's generator and
// never use what they draw (ShiftMapping.slang:90,105,183,253,301,377), so every
// shift result is independent of the generator state.  The per-pixel loop of the
// reference is therefore split into one kernel per shift kind, each thread doing
// one shift of one kind (coherent code, small register footprint, one thread per
// splat instead of a per-pixel loop of variable length), followed by a combine
// kernel that replays the reference's resampling order (and its generator draws)
// on the stored results with no ray queries.  Results are identical to the
// single-kernel form; only the schedule changes.
#pragma once
#include "kernels.h"

namespace rs {

__device__ __forceinline__ void store_shift(const ShiftPlanes& P, size_t i, const Shifted& s)
{
    uint4* p = P.p + i;
    const size_t st = P.stride;
    p[0] = make_uint4(f2u(s.radiance.x), f2u(s.radiance.y), f2u(s.radiance.z), f2u(s.subPixelJacobian));
    p[st] = make_uint4(f2u(s.lensVertexJacobian), f2u(s.secondaryPathJacobian), f2u(s.fractionalPixel.x), f2u(s.fractionalPixel.y));
    p[2 * st] = make_uint4(s.primaryHit.w[0], s.primaryHit.w[1], s.primaryHit.w[2], s.primaryHit.w[3]);
    p[3 * st] = make_uint4(f2u(s.lensSample.x), f2u(s.lensSample.y), f2u(s.firstRayDir.x), f2u(s.firstRayDir.y));
    p[4 * st] = make_uint4(f2u(s.firstRayDir.z), 0u, 0u, 0u);
}
__device__ __forceinline__ Shifted load_shift(const ShiftPlanes& P, size_t i)
{
    const uint4* p = P.p + i;
    const size_t st = P.stride;
    uint4 a = __ldg(p), b = __ldg(p + st), c = __ldg(p + 2 * st), d = __ldg(p + 3 * st), e = __ldg(p + 4 * st);
    Shifted s;
    s.radiance = mk3(u2f(a.x), u2f(a.y), u2f(a.z));
    s.subPixelJacobian = u2f(a.w);
    s.lensVertexJacobian = u2f(b.x);
    s.secondaryPathJacobian = u2f(b.y);
    s.fractionalPixel = mk2(u2f(b.z), u2f(b.w));
    s.primaryHit.w[0] = c.x; s.primaryHit.w[1] = c.y; s.primaryHit.w[2] = c.z; s.primaryHit.w[3] = c.w;
    s.lensSample = mk2(u2f(d.x), u2f(d.y));
    s.firstRayDir = mk3(u2f(d.z), u2f(d.w), u2f(e.x));
    return s;
}

// The backup (gathered) reservoir of pixel (x, y) with the Clamped gather: the previous
// frame's reservoir at round(prevPixel) (CollectTemporalSamples.cs.slang:84-99, 143-156).
// Returns its index in the previous frame or kInvalidIndex, and the floating coordinate.
__device__ __forceinline__ uint32_t clamped_backup(const DevCtx& C, const float2* mvec, uint32_t x, uint32_t y, f2& floatingCoord)
{
    float2 m = __ldg(&mvec[y * C.W + x]);
    f2 mv = mk2(m.x, m.y);
    mv = (length(mv) < 1e-06f) ? mk2(0.f, 0.f) : mv;
    f2 prevPixel = mk2((float)x + mv.x * (float)C.W, (float)y + mv.y * (float)C.H);
    floatingCoord = mk2(-1.f, -1.f);
    if (!valid_float(C, prevPixel)) return kInvalidIndex;
    float rx = f_round(prevPixel.x), ry = f_round(prevPixel.y);
    floatingCoord = mk2(rx, ry);
    if (!valid_int(C, (int)rx, (int)ry)) return kInvalidIndex;
    return (uint32_t)ry * C.W + (uint32_t)rx;
}

__device__ __forceinline__ void backup_of(const DevCtx& C, const WaveCtx& K, uint32_t ri, uint32_t x, uint32_t y, Res& br, uint32_t& bi, f2& fc)
{
    if (K.fused)
    {
        bi = clamped_backup(C, K.mvec, x, y, fc);
        br = bi != kInvalidIndex ? load_res(K.prev, bi) : res_default();
        if (f_isnan(br.totalWeight)) { br.integrand = mk3(0.f); br.totalWeight = 0.f; }
    }
    else
    {
        bi = ri;
        br = load_res(K.inter, ri);
        float2 f = __ldg(&K.floatingCoords[ri]);
        fc = mk2(f.x, f.y);
    }
}

__device__ __forceinline__ Recon backup_rec(const WaveCtx& K, uint32_t bi)
{
    if (!K.fused) return load_rec(K.interRec, bi);
    if (bi == kInvalidIndex) return recon_default();
    Recon r = load_rec(K.prevRec, bi);
    Res br = load_res(K.prev, bi);
    if (f_isnan(br.totalWeight))
    {
        r.subPixelJacobian = 1.f; r.lensVertexJacobian = 1.f; r.secondaryPathJacobian = 1.f; r.pathLength = 0;
    }
    return r;
}

// ================================================================ ScatterOnly
// ScatterTemporalResampling.rt.slang:65-174: the current sample's reprojection shift into the
// previous frame (k_so_curr) and every splat's reprojection shift into its cell (k_so_splat, one
// thread per splat of the sorted cell lists) are stored; the combine walks each cell's splats in the
// canonical order and replays the resampling draws.  Buffers: m2curr, splatShift / splatTerms
// (prevPHat, Jacobian) / splatM (MIS weight, 0, shifted sub-pixel).
template <bool kEnv>
__global__ void __launch_bounds__(128, 8) k_so_curr(uint32_t slot, WaveCtx K)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const f3 integrand = load_integrand(K.curr, ri);
    if (!any_gt0(integrand)) return;
    const Recon crd = load_rec(K.currRec, ri);
    SampleGen dummy = {0, C.sgKind};
    Shifted sc = dev_scatter_shift<kEnv>(C, dummy, crd, crd.time + C.cm.artificialFrameTime, crd.firstHit, crd.lensSample, false);
    float sj = jac_scatter(sc, crd);
    float m2 = luminance(sc.radiance) * sj;
    m2 = f_isnan(m2) ? 0.f : m2;
    int spx = (int)f_floor(sc.fractionalPixel.x), spy = (int)f_floor(sc.fractionalPixel.y);
    if (valid_int(C, spx, spy)) m2 *= C.useConfTemporal ? load_confidence(K.prev, (uint32_t)spy * C.W + (uint32_t)spx) : 1.f;
    else m2 = 0.f;
    K.m2curr[ri] = m2;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 8) k_so_splat(uint32_t slot, WaveCtx K)
{
    const DevCtx& C = c_ctx[slot];
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= *K.totalSplats) return;
    const uint32_t si = __ldg(&K.sorted[j]);
    const Res pr = load_res(K.prev, si);
    if (!any_gt0(pr.integrand)) return;
    const uint32_t cell = __ldg(&K.sortedCell[j]);
    const Recon prd = load_rec(K.prevRec, si);
    SampleGen dummy = {0, C.sgKind};
    Shifted sp = dev_scatter_shift<kEnv>(C, dummy, prd, prd.time, prd.firstHit, prd.lensSample, false);
    store_shift(K.splatShift, j, sp);
    float sj = jac_scatter(sp, prd);
    const float m1 = luminance(sp.radiance) * sj * (C.useConfTemporal ? load_confidence(K.curr, cell) : 1.f);
    const f3 prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
    sj = f_isnan(m1) ? 1.f : sj;
    const float m2 = luminance(pr.integrand) * (C.useConfTemporal ? pr.confidence : 1.f);
    const float prevSampleMIS = ((m1 + m2) == 0.f) ? 0.f : m2 / (m1 + m2);
    const f2 sub = sp.fractionalPixel - floor2(sp.fractionalPixel); // recon_update's sub-pixel
    K.splatTerms[j] = make_float4(prevPHat.x, prevPHat.y, prevPHat.z, sj);
    K.splatM[j] = make_float4(prevSampleMIS, 0.f, sub.x, sub.y);
}

__global__ void __launch_bounds__(128) k_so_combine(uint32_t slot, WaveCtx K, float4* __restrict__ color)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const uint32_t x = ri % C.W, y = ri / C.W;
    const bool useConf = C.useConfTemporal != 0;
    SampleGen sg = sg_create(x, y, pass_seed(C, 5), C.sgKind);
    Res dst = res_default();
    Recon dstR = recon_default();
    const Res cr = load_res_rw(K.curr, ri);
    float currSampleMIS = 1.f;
    if (any_gt0(cr.integrand))
    {
        const float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
        const float m2 = K.m2curr[ri];
        currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
    }
    if (res_add_sample(dst, sg, currSampleMIS, cr.integrand, 1.f, cr)) dstR = load_rec_rw(K.currRec, ri);
    const float newConfidence = dst.confidence;
    const uint32_t n = __ldg(&K.counts[ri]), off = __ldg(&K.offsets[ri]);
    for (uint32_t i = 0; i < n; i++)
    {
        const uint32_t j = off + i;
        const uint32_t si = __ldg(&K.sorted[j]);
        Res pr = load_res(K.prev, si);
        float prevSampleMIS = 0.f;
        f3 prevPHat = mk3(0.f);
        float sj = 1.f;
        const bool shifted = any_gt0(pr.integrand);
        if (shifted)
        {
            const float4 t = __ldg(&K.splatTerms[j]);
            const float4 m = __ldg(&K.splatM[j]);
            prevPHat = mk3(t.x, t.y, t.z);
            sj = t.w;
            prevSampleMIS = m.x;
            pr.subPixel = mk2(m.z, m.w);
        }
        if (res_add_sample(dst, sg, prevSampleMIS, prevPHat, sj, pr))
        {
            dstR = load_rec(K.prevRec, si);
            if (shifted) recon_update(dstR, load_shift(K.splatShift, j));
        }
    }
    dst.confidence = bilinear_confidence(C, K.mvec, K.prev, x, y, newConfidence, useConf);
    store_res(K.curr, ri, dst);
    store_rec(K.currRec, ri, dstR);
    write_color(color, ri, dst);
}

// ================================================================ GatherOnly, lens-copy stage
// GatherTemporalResampling.rt.slang:68-235 without depth of field (the lens-copy stage alone, with
// probability 1): the current sample's shift into the previous frame and the gathered sample's shift
// into this pixel are independent kernels (their generator copies are never used), the combine
// replays the pixel's two resampling draws.  Buffers: m2curr (the current sample's MIS term),
// backupShift / backupTerms / backupM (the gathered sample's shift, prevPHat and Jacobian, MIS term).
template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_go_curr(uint32_t slot, WaveCtx K)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const Res cr = load_res(K.curr, ri);
    if (!any_gt0(cr.integrand)) return;
    const Res pr = load_res(K.inter, ri);
    const float2 fcv = __ldg(&K.floatingCoords[ri]);
    const Recon crd = load_rec(K.currRec, ri);
    SampleGen dummy = {0, C.sgKind};
    Shifted sc = dev_gather_lens_copy<kEnv>(C, dummy, crd, crd.time + C.cm.artificialFrameTime, mk2(fcv.x, fcv.y) + cr.subPixel, crd.lensSample);
    float sj = sc.secondaryPathJacobian / crd.secondaryPathJacobian;
    float m2 = luminance(sc.radiance) * sj * (C.useConfTemporal ? pr.confidence : 1.f) * 1.f;
    K.m2curr[ri] = f_isnan(m2) ? 0.f : m2;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_go_prev(uint32_t slot, WaveCtx K)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const Res pr = load_res(K.inter, ri);
    if (!any_gt0(pr.integrand)) return;
    const uint32_t x = ri % C.W, y = ri / C.W;
    const Res cr = load_res(K.curr, ri);
    const Recon prd = load_rec(K.interRec, ri);
    SampleGen dummy = {0, C.sgKind};
    Shifted sp = dev_gather_lens_copy<kEnv>(C, dummy, prd, prd.time, mk2((float)x + pr.subPixel.x, (float)y + pr.subPixel.y), prd.lensSample);
    store_shift(K.backupShift, ri, sp);
    float sj = sp.secondaryPathJacobian / prd.secondaryPathJacobian;
    float m1 = luminance(sp.radiance) * sj * (C.useConfTemporal ? cr.confidence : 1.f);
    const f3 prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
    sj = f_isnan(m1) ? 1.f : sj;
    m1 = f_isnan(m1) ? 0.f : m1;
    K.backupTerms[ri] = make_float4(prevPHat.x, prevPHat.y, prevPHat.z, sj);
    K.backupM[ri] = make_float2(m1, 0.f);
}

__global__ void __launch_bounds__(128) k_go_combine(uint32_t slot, WaveCtx K, float4* __restrict__ color)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const uint32_t x = ri % C.W, y = ri / C.W;
    const bool useConf = C.useConfTemporal != 0;
    SampleGen sg = sg_create(x, y, pass_seed(C, 3), C.sgKind);
    Res dst = res_default();
    Recon dstR = recon_default();
    const Res cr = load_res_rw(K.curr, ri);
    const Res pr = load_res(K.inter, ri);
    float currSampleMIS = 0.f;
    f3 currPHat = mk3(0.f);
    if (any_gt0(cr.integrand))
    {
        const float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
        currPHat = cr.integrand;
        const float m2 = K.m2curr[ri];
        currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
    }
    if (res_add_sample(dst, sg, currSampleMIS, currPHat, 1.f, cr)) dstR = load_rec_rw(K.currRec, ri);
    float prevSampleMIS = 0.f;
    f3 prevPHat = mk3(0.f);
    float sj = 1.f;
    if (any_gt0(pr.integrand))
    {
        const float4 t = __ldg(&K.backupTerms[ri]);
        prevPHat = mk3(t.x, t.y, t.z);
        sj = t.w;
        const float m1 = __ldg(&K.backupM[ri]).x;
        const float m2 = luminance(pr.integrand) * (useConf ? pr.confidence : 1.f) * 1.f;
        prevSampleMIS = ((m1 + m2) == 0.f) ? 0.f : m2 / (m1 + m2);
    }
    if (res_add_sample(dst, sg, prevSampleMIS, prevPHat, sj, pr))
    {
        dstR = load_rec(K.interRec, ri);
        recon_update(dstR, load_shift(K.backupShift, ri));
    }
    store_res(K.curr, ri, dst);
    store_rec(K.currRec, ri, dstR);
    write_color(color, ri, dst);
}

// ---- stage 1: current sample -> previous domain by reprojection (ScatterBackup...:96-114)
template <bool kEnv>
__device__ __forceinline__ void sb_curr_scatter_body(uint32_t slot, const WaveCtx& K, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel_at(C.W, C.H, blk, ri)) return;
    f3 integrand = load_integrand(K.curr, ri);
    if (!any_gt0(integrand)) return;
    Recon crd = load_rec_rw(K.currRec, ri);
    SampleGen dummy = {0, C.sgKind};
    Shifted sc = dev_scatter_shift<kEnv>(C, dummy, crd, crd.time + C.cm.artificialFrameTime, crd.firstHit, crd.lensSample, false);
    float scj = jac_scatter(sc, crd);
    float m2 = luminance(sc.radiance) * scj;
    m2 = f_isnan(m2) ? 0.f : m2;
    int spx = (int)f_floor(sc.fractionalPixel.x), spy = (int)f_floor(sc.fractionalPixel.y);
    if (valid_int(C, spx, spy)) m2 *= 0.5f * (C.useConfTemporal ? load_confidence(K.prev, (uint32_t)spy * C.W + (uint32_t)spx) : 1.f);
    else m2 = 0.f;
    K.m2curr[ri] = m2;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 8) k_sb_curr_scatter(uint32_t slot, WaveCtx K)
{
    sb_curr_scatter_body<kEnv>(slot, K, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 8) kb_sb_curr_scatter(BatchQueue q, const WaveCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveCtx& a = args[inst];
        sb_curr_scatter_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

// ---- stage 1: current sample -> previous domain by the gather shift (:116-129)
template <bool kEnv>
__device__ __forceinline__ void sb_curr_gather_body(uint32_t slot, const WaveCtx& K, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel_at(C.W, C.H, blk, ri)) return;
    Res cr = load_res_rw(K.curr, ri);
    if (!any_gt0(cr.integrand)) return;
    uint32_t x = ri % C.W, y = ri / C.W;
    Res br; uint32_t bi; f2 fc;
    backup_of(C, K, ri, x, y, br, bi, fc);
    float m3 = 0.f;
    if (valid_float(C, fc))
    {
        Recon crd = load_rec_rw(K.currRec, ri);
        SampleGen dummy = {0, C.sgKind};
        Shifted gc = dev_gather_lens_copy<kEnv>(C, dummy, crd, crd.time + C.cm.artificialFrameTime, fc + cr.subPixel, crd.lensSample);
        float gj = gc.secondaryPathJacobian / crd.secondaryPathJacobian;
        m3 = luminance(gc.radiance) * gj * 0.5f * (C.useConfTemporal ? br.confidence : 1.f);
    }
    m3 = f_isnan(m3) ? 0.f : m3;
    K.m3curr[ri] = m3;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_sb_curr_gather(uint32_t slot, WaveCtx K)
{
    sb_curr_gather_body<kEnv>(slot, K, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) kb_sb_curr_gather(BatchQueue q, const WaveCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveCtx& a = args[inst];
        sb_curr_gather_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

// ---- stage 1: backup sample -> current domain (:156-166)
template <bool kEnv>
__device__ __forceinline__ void sb_backup_gather_body(uint32_t slot, const WaveCtx& K, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel_at(C.W, C.H, blk, ri)) return;
    uint32_t x = ri % C.W, y = ri / C.W;
    Res br; uint32_t bi; f2 fc;
    backup_of(C, K, ri, x, y, br, bi, fc);
    if (!any_gt0(br.integrand)) return;
    Recon brd = backup_rec(K, bi);
    SampleGen dummy = {0, C.sgKind};
    Shifted sb = dev_gather_lens_copy<kEnv>(C, dummy, brd, brd.time, mk2((float)x + br.subPixel.x, (float)y + br.subPixel.y), brd.lensSample);
    store_shift(K.backupShift, ri, sb);
    float sj = sb.secondaryPathJacobian / brd.secondaryPathJacobian;
    float currConf = load_confidence(K.curr, ri);
    float m1 = luminance(sb.radiance) * sj * (C.useConfTemporal ? currConf : 1.f);
    f3 backupPHat = f_isnan(m1) ? mk3(0.f) : sb.radiance;
    sj = f_isnan(m1) ? 1.f : sj;
    m1 = f_isnan(m1) ? 0.f : m1;
    K.backupTerms[ri] = make_float4(backupPHat.x, backupPHat.y, backupPHat.z, sj);
    K.backupM[ri] = make_float2(m1, 0.f);
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_sb_backup_gather(uint32_t slot, WaveCtx K)
{
    sb_backup_gather_body<kEnv>(slot, K, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) kb_sb_backup_gather(BatchQueue q, const WaveCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveCtx& a = args[inst];
        sb_backup_gather_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

// ---- stage 2 (Balance): updated backup -> previous domain by reprojection (:171-189)
template <bool kEnv>
__device__ __forceinline__ void sb_backup_scatter_body(uint32_t slot, const WaveCtx& K, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel_at(C.W, C.H, blk, ri)) return;
    uint32_t x = ri % C.W, y = ri / C.W;
    Res br; uint32_t bi; f2 fc;
    backup_of(C, K, ri, x, y, br, bi, fc);
    if (!any_gt0(br.integrand)) return;
    Recon brd = backup_rec(K, bi);
    Shifted sb = load_shift(K.backupShift, ri);
    recon_update(brd, sb);
    float sj = __ldg(&K.backupTerms[ri]).w;
    SampleGen dummy = {0, C.sgKind};
    Shifted ss = dev_scatter_shift<kEnv>(C, dummy, brd, brd.time + C.cm.artificialFrameTime, brd.firstHit, brd.lensSample, false);
    float scj = jac_scatter(ss, brd);
    float m2 = luminance(ss.radiance) * scj * sj;
    m2 = f_isnan(m2) ? 0.f : m2;
    int spx = (int)f_floor(ss.fractionalPixel.x), spy = (int)f_floor(ss.fractionalPixel.y);
    if (valid_int(C, spx, spy)) m2 *= 0.5f * (C.useConfTemporal ? load_confidence(K.prev, (uint32_t)spy * C.W + (uint32_t)spx) : 1.f);
    else m2 = 0.f;
    K.backupM[ri].y = m2;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 8) k_sb_backup_scatter(uint32_t slot, WaveCtx K)
{
    sb_backup_scatter_body<kEnv>(slot, K, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 8) kb_sb_backup_scatter(BatchQueue q, const WaveCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveCtx& a = args[inst];
        sb_backup_scatter_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

// ---- stage 1: splatted previous sample -> current domain (:218-235), one thread per splat
template <bool kEnv>
__device__ __forceinline__ void sb_splat_scatter_body(uint32_t slot, const WaveCtx& K, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t j = blk.b * blockDim.x + threadIdx.x;
    if (j >= *K.totalSplats) return;
    uint32_t si = __ldg(&K.sorted[j]);
    uint32_t cell = __ldg(&K.sortedCell[j]);
    f3 integrand = load_integrand(K.prev, si);
    if (!any_gt0(integrand)) return;
    Recon prd = load_rec(K.prevRec, si);
    SampleGen dummy = {0, C.sgKind};
    Shifted sp = dev_scatter_shift<kEnv>(C, dummy, prd, prd.time, prd.firstHit, prd.lensSample, true);
    store_shift(K.splatShift, j, sp);
    float scj = jac_scatter(sp, prd);
    float m1 = luminance(sp.radiance) * scj * (C.useConfTemporal ? load_confidence(K.curr, cell) : 1.f);
    m1 = f_isnan(m1) ? 0.f : m1;
    // The NaN tests of :225-226 see the already cleared m1, so prevPHat and the Jacobian pass unchanged.
    f2 sub = sp.fractionalPixel - floor2(sp.fractionalPixel);
    K.splatTerms[j] = make_float4(sp.radiance.x, sp.radiance.y, sp.radiance.z, scj);
    K.splatM[j] = make_float4(m1, 0.f, sub.x, sub.y);
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_sb_splat_scatter(uint32_t slot, WaveCtx K)
{
    sb_splat_scatter_body<kEnv>(slot, K, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) kb_sb_splat_scatter(BatchQueue q, const WaveCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveCtx& a = args[inst];
        sb_splat_scatter_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

// ---- stage 2 (Balance): updated splat -> previous domain by the gather shift (:237-253)
template <bool kEnv>
__device__ __forceinline__ void sb_splat_gather_body(uint32_t slot, const WaveCtx& K, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t j = blk.b * blockDim.x + threadIdx.x;
    if (j >= *K.totalSplats) return;
    uint32_t si = __ldg(&K.sorted[j]);
    f3 integrand = load_integrand(K.prev, si);
    if (!any_gt0(integrand)) return;
    uint32_t cell = __ldg(&K.sortedCell[j]);
    uint32_t x = cell % C.W, y = cell / C.W;
    Res br; uint32_t bi; f2 fc;
    backup_of(C, K, cell, x, y, br, bi, fc);
    float4 sm = __ldg(&K.splatM[j]);
    f2 fp = fc + mk2(sm.z, sm.w);
    float m3 = 0.f;
    if (valid_float(C, fp))
    {
        Recon prd = load_rec(K.prevRec, si);
        Shifted sp = load_shift(K.splatShift, j);
        recon_update(prd, sp);
        float scj = __ldg(&K.splatTerms[j]).w;
        SampleGen dummy = {0, C.sgKind};
        Shifted gp = dev_gather_lens_copy<kEnv>(C, dummy, prd, prd.time + C.cm.artificialFrameTime, fp, prd.lensSample);
        float gj = gp.secondaryPathJacobian / prd.secondaryPathJacobian;
        m3 = luminance(gp.radiance) * gj * scj * 0.5f * (C.useConfTemporal ? br.confidence : 1.f);
    }
    m3 = f_isnan(m3) ? 0.f : m3;
    K.splatM[j].y = m3;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_sb_splat_gather(uint32_t slot, WaveCtx K)
{
    sb_splat_gather_body<kEnv>(slot, K, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) kb_sb_splat_gather(BatchQueue q, const WaveCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveCtx& a = args[inst];
        sb_splat_gather_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

// ---- combine: the GRIS order of ScatterBackupTemporalResampling.rt.slang:91-283 on stored shifts
__device__ __forceinline__ void sb_combine_body(uint32_t slot, const WaveCtx& K, float4* __restrict__ color, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel_at(C.W, C.H, blk, ri)) return;
    uint32_t x = ri % C.W, y = ri / C.W;
    const bool useConf = C.useConfTemporal != 0;
    const bool balance = C.scatterBackupMIS == 0u;
    const float misScale = balance ? 1.f : 0.5f;
    SampleGen sg = sg_create(x, y, pass_seed(C, 6), C.sgKind);
    Res dst = res_default();
    Res cr = load_res_rw(K.curr, ri);
    Res br; uint32_t bi; f2 fc;
    backup_of(C, K, ri, x, y, br, bi, fc);
    enum { kSelNone = 0, kSelCurr = 1, kSelBackup = 2, kSelSplat = 3 };
    uint32_t sel = kSelNone, selIndex = 0;
    {
        float currSampleMIS = 1.f;
        if (any_gt0(cr.integrand))
        {
            float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
            float m2 = K.m2curr[ri];
            float m3 = K.m3curr[ri];
            if (balance) currSampleMIS = (m1 + m2 + m3 == 0.f) ? 0.f : m1 / (m1 + m2 + m3);
            else currSampleMIS = 0.5f * (((m1 + m2 == 0.f) ? 0.f : 0.5f * m1 / (0.5f * m1 + m2)) +
                                         ((m1 + m3 == 0.f) ? 0.f : 0.5f * m1 / (0.5f * m1 + m3)));
        }
        if (res_add_sample(dst, sg, currSampleMIS, cr.integrand, 1.f, cr)) sel = kSelCurr;
    }
    {
        float backupSampleMIS = 0.f;
        f3 backupPHat = mk3(0.f);
        float sj = 1.f;
        if (any_gt0(br.integrand))
        {
            float4 bt = __ldg(&K.backupTerms[ri]);
            float2 bm = __ldg(&K.backupM[ri]);
            backupPHat = mk3(bt.x, bt.y, bt.z);
            sj = bt.w;
            float m1 = bm.x;
            float m2 = balance ? bm.y : 0.f;
            float m3 = luminance(br.integrand) * 0.5f * (useConf ? br.confidence : 1.f);
            backupSampleMIS = misScale * ((m1 + m2 + m3 == 0.f) ? 0.f : m3 / (misScale * m1 + m2 + m3));
        }
        if (res_add_sample(dst, sg, backupSampleMIS, backupPHat, sj, br)) sel = kSelBackup;
    }
    float newConfidence = dst.confidence;
    uint32_t n = K.counts[ri], off = K.offsets[ri];
    for (uint32_t i = 0; i < n; i++)
    {
        uint32_t j = off + i;
        uint32_t si = __ldg(&K.sorted[j]);
        Res pr = load_res(K.prev, si);
        float prevSampleMIS = 0.f;
        f3 prevPHat = mk3(0.f);
        float scj = 1.f;
        if (any_gt0(pr.integrand))
        {
            float4 st = __ldg(&K.splatTerms[j]);
            float4 sm = __ldg(&K.splatM[j]);
            prevPHat = mk3(st.x, st.y, st.z);
            scj = st.w;
            float m1 = sm.x;
            pr.subPixel = mk2(sm.z, sm.w);
            float m2 = luminance(pr.integrand) * 0.5f * (useConf ? pr.confidence : 1.f);
            float m3 = balance ? sm.y : 0.f;
            prevSampleMIS = misScale * ((m1 + m2 + m3 == 0.f) ? 0.f : m2 / (misScale * m1 + m2 + m3));
        }
        if (res_add_sample(dst, sg, prevSampleMIS, prevPHat, scj, pr)) { sel = kSelSplat; selIndex = j; }
    }
    // bilinear confidence (ScatterBackupTemporalResampling.rt.slang:262-279)
    {
        float2 m = __ldg(&K.mvec[ri]);
        f2 mv = mk2(m.x, m.y);
        mv = (length(mv) < 1e-06f) ? mk2(0.f, 0.f) : mv;
        f2 prevPixel = mk2((float)x + mv.x * (float)C.W, (float)y + mv.y * (float)C.H);
        int tlx = (int)f_floor(prevPixel.x), tly = (int)f_floor(prevPixel.y);
        f2 frac = mk2(f_saturate(prevPixel.x - (float)tlx), f_saturate(prevPixel.y - (float)tly));
        for (int ox = 0; ox < 2; ox++)
            for (int oy = 0; oy < 2; oy++)
            {
                int nx = tlx + ox, ny = tly + oy;
                if (!valid_int(C, nx, ny)) continue;
                float bw = f_lerp((float)(1 - ox), (float)ox, frac.x) * f_lerp((float)(1 - oy), (float)oy, frac.y);
                newConfidence += bw * (useConf ? load_confidence(K.prev, (uint32_t)ny * C.W + (uint32_t)nx) : 1.f);
            }
        dst.confidence = f_min(kConfidenceCap, newConfidence);
    }
    store_res(K.curr, ri, dst);
    // The selected sample's reconnection record: the current one is already in place.
    if (sel == kSelBackup)
    {
        Recon brd = backup_rec(K, bi);
        recon_update(brd, load_shift(K.backupShift, ri));
        store_rec(K.currRec, ri, brd);
    }
    else if (sel == kSelSplat)
    {
        Recon prd = load_rec(K.prevRec, __ldg(&K.sorted[selIndex]));
        recon_update(prd, load_shift(K.splatShift, selIndex));
        store_rec(K.currRec, ri, prd);
    }
    else if (sel == kSelNone)
    {
        store_rec(K.currRec, ri, recon_default());
    }
    if (color)
    {
        f3 c = dst.integrand * res_ucw(dst);
        color[ri] = make_float4(c.x, c.y, c.z, 1.f);
    }
}

__global__ void __launch_bounds__(128) k_sb_combine(uint32_t slot, WaveCtx K, float4* __restrict__ color)
{
    sb_combine_body(slot, K, color, Blk{blockIdx.x, 8u});
}

__global__ void __launch_bounds__(128) kb_sb_combine(BatchQueue q, const WaveColorArgs* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const WaveColorArgs& a = args[inst];
        sb_combine_body(__ldg(q.slot + inst), a.K, a.color, batch_blk(q, inst, t));
    }
}

// ============================================================ spatial resampling, wavefront form
// Per (pixel, neighbour slot i): the central -> neighbour shift (m1) and the neighbour -> central
// shift (SpatialResampling.rt.slang:110-174).  The start index of the neighbour sequence is the
// pixel generator's first draw, recomputed here.
__device__ __forceinline__ bool spatial_neighbor(const DevCtx& C, uint32_t iteration, const float2* neighborOffsets, uint32_t x, uint32_t y,
                                                 uint32_t i, int& nx, int& ny)
{
    SampleGen sg = sg_create(x, y, C.useFixedSeed ? C.fixedSeed + 7 : kNumRenderPasses * (C.frameCount + C.seed) + 1337u * iteration + 7u, C.sgKind);
    uint32_t startIdx = (uint32_t)(sampleNext1D(sg) * 8192.f);
    float2 off = __ldg(&neighborOffsets[(startIdx + i) % 8192u]);
    nx = (int)f_round((float)x + C.spatialGatherRadius * off.x);
    ny = (int)f_round((float)y + C.spatialGatherRadius * off.y);
    return valid_int(C, nx, ny);
}

template <bool kEnv>
__device__ __forceinline__ void sp_central_body(uint32_t slot, const SpatialCtx& S, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    // blockIdx.y: the neighbour; blockIdx.x / threadIdx.x: the pixel (tiled)
    const uint32_t N = C.W * C.H;
    uint32_t ri;
    if (blockIdx.y >= C.neighborCount || !tiled_pixel_at(C.W, C.H, blk, ri)) return;
    const uint32_t i = blockIdx.y, t = i * N + ri;
    uint32_t x = ri % C.W, y = ri / C.W;
    int nx, ny;
    if (!spatial_neighbor(C, S.iteration, S.neighborOffsets, x, y, i, nx, ny)) return;
    Res cent = load_res(S.src, ri);
    float m1 = 0.f;
    if (any_gt0(cent.integrand))
    {
        f2 probs = pixel_dof_probs(C, S.vbuffer, ri);
        const bool lensCopy = i < (uint32_t)f_round(probs.x * (float)C.neighborCount);
        Recon centR = load_rec(S.srcRec, ri);
        uint32_t ni = (uint32_t)ny * C.W + (uint32_t)nx;
        f2 fp = mk2((float)nx + cent.subPixel.x, (float)ny + cent.subPixel.y);
        SampleGen dummy = {0, C.sgKind};
        Shifted sc = lensCopy ? dev_gather_lens_copy<kEnv>(C, dummy, centR, centR.time, fp, centR.lensSample)
                              : dev_gather_primary_reconnect<kEnv>(C, dummy, centR, centR.time, fp, centR.firstHit);
        float sj = (lensCopy ? 1.f : (sc.lensVertexJacobian / centR.lensVertexJacobian)) * (sc.secondaryPathJacobian / centR.secondaryPathJacobian);
        m1 = luminance(sc.radiance) * sj * (C.useConfSpatial ? load_confidence(S.src, ni) : 1.f);
        m1 = f_isnan(m1) ? 0.f : m1;
    }
    S.m1[t] = m1;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 10) k_sp_central(uint32_t slot, SpatialCtx S)
{
    sp_central_body<kEnv>(slot, S, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 10) kb_sp_central(BatchQueue q, const SpatialCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const SpatialCtx& a = args[inst];
        sp_central_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

template <bool kEnv>
__device__ __forceinline__ void sp_neighbor_body(uint32_t slot, const SpatialCtx& S, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    // blockIdx.y: the neighbour; blockIdx.x / threadIdx.x: the pixel (tiled)
    const uint32_t N = C.W * C.H;
    uint32_t ri;
    if (blockIdx.y >= C.neighborCount || !tiled_pixel_at(C.W, C.H, blk, ri)) return;
    const uint32_t i = blockIdx.y, t = i * N + ri;
    uint32_t x = ri % C.W, y = ri / C.W;
    int nx, ny;
    if (!spatial_neighbor(C, S.iteration, S.neighborOffsets, x, y, i, nx, ny)) return;
    uint32_t ni = (uint32_t)ny * C.W + (uint32_t)nx;
    Res nr = load_res(S.src, ni);
    if (!any_gt0(nr.integrand)) return;
    f2 probs = pixel_dof_probs(C, S.vbuffer, ri);
    const bool lensCopy = i < (uint32_t)f_round(probs.x * (float)C.neighborCount);
    Recon nrd = load_rec(S.srcRec, ni);
    f2 fp = mk2((float)x + nr.subPixel.x, (float)y + nr.subPixel.y);
    SampleGen dummy = {0, C.sgKind};
    Shifted sn = lensCopy ? dev_gather_lens_copy<kEnv>(C, dummy, nrd, nrd.time, fp, nrd.lensSample)
                          : dev_gather_primary_reconnect<kEnv>(C, dummy, nrd, nrd.time, fp, nrd.firstHit);
    store_shift(S.shift, t, sn);
    float sj = (lensCopy ? 1.f : (sn.lensVertexJacobian / nrd.lensVertexJacobian)) * (sn.secondaryPathJacobian / nrd.secondaryPathJacobian);
    float nw = luminance(sn.radiance) * sj * (C.useConfSpatial ? load_confidence(S.src, ri) : 1.f);
    f3 neighborPHat = f_isnan(nw) ? mk3(0.f) : sn.radiance;
    sj = f_isnan(nw) ? 1.f : sj;
    nw = f_isnan(nw) ? 0.f : nw / (float)C.neighborCount;
    S.terms[t] = make_float4(neighborPHat.x, neighborPHat.y, neighborPHat.z, sj);
    S.nw[t] = nw;
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) k_sp_neighbor(uint32_t slot, SpatialCtx S)
{
    sp_neighbor_body<kEnv>(slot, S, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 9) kb_sp_neighbor(BatchQueue q, const SpatialCtx* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const SpatialCtx& a = args[inst];
        sp_neighbor_body<kEnv>(__ldg(q.slot + inst), a, batch_blk(q, inst, t));
    }
}

__device__ __forceinline__ void sp_combine_body(uint32_t slot, const SpatialCtx& S, float4* __restrict__ color, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    const uint32_t N = C.W * C.H;
    if (!tiled_pixel_at(C.W, C.H, blk, ri)) return;
    uint32_t x = ri % C.W, y = ri / C.W;
    const bool useConf = C.useConfSpatial != 0;
    const uint32_t neighborCount = C.neighborCount;
    SampleGen sg = sg_create(x, y, C.useFixedSeed ? C.fixedSeed + 7 : kNumRenderPasses * (C.frameCount + C.seed) + 1337u * S.iteration + 7u, C.sgKind);
    Res cent = load_res(S.src, ri);
    float centralSampleMIS = 1.f;
    float centralWeight = luminance(cent.integrand) / (float)neighborCount * (useConf ? cent.confidence : 1.f);
    Res dst = res_default();
    int validNeighbors = 0;
    uint32_t startIdx = (uint32_t)(sampleNext1D(sg) * 8192.f);
    uint32_t sel = kInvalidIndex; // slot index t of the selected neighbour, or N * count for the central sample
    for (uint32_t i = 0; i < neighborCount; i++)
    {
        float2 off = __ldg(&S.neighborOffsets[(startIdx + i) % 8192u]);
        int nx = (int)f_round((float)x + C.spatialGatherRadius * off.x);
        int ny = (int)f_round((float)y + C.spatialGatherRadius * off.y);
        if (!valid_int(C, nx, ny)) continue;
        validNeighbors += 1;
        uint32_t t = i * N + ri;
        uint32_t ni = (uint32_t)ny * C.W + (uint32_t)nx;
        Res nr = load_res(S.src, ni);
        float m1 = any_gt0(cent.integrand) ? __ldg(&S.m1[t]) : 0.f;
        centralSampleMIS += 1.f;
        centralSampleMIS -= (m1 + centralWeight > 0.f) ? m1 / (m1 + centralWeight) : 0.f;
        float neighborSampleMIS = 0.f;
        f3 neighborPHat = mk3(0.f);
        float sj = 1.f;
        if (any_gt0(nr.integrand))
        {
            float4 tm = __ldg(&S.terms[t]);
            neighborPHat = mk3(tm.x, tm.y, tm.z);
            sj = tm.w;
            float nw = __ldg(&S.nw[t]);
            float m2 = luminance(nr.integrand) * (useConf ? nr.confidence : 1.f);
            neighborSampleMIS = (m2 + nw > 0.f) ? m2 / (nw + m2) : 0.f;
        }
        if (res_add_sample(dst, sg, neighborSampleMIS, neighborPHat, sj, nr)) sel = t;
    }
    if (res_add_sample(dst, sg, centralSampleMIS, cent.integrand, 1.f, cent)) sel = N * neighborCount;
    dst.totalWeight /= (float)(validNeighbors + 1);
    store_res(S.dst, ri, dst);
    Recon out;
    if (sel == N * neighborCount) out = load_rec(S.srcRec, ri);
    else if (sel != kInvalidIndex)
    {
        uint32_t i = sel / N;
        int nx, ny;
        spatial_neighbor(C, S.iteration, S.neighborOffsets, x, y, i, nx, ny);
        out = load_rec(S.srcRec, (uint32_t)ny * C.W + (uint32_t)nx);
        recon_update(out, load_shift(S.shift, sel));
    }
    else out = recon_default();
    store_rec(S.dstRec, ri, out);
    if (color)
    {
        f3 c = dst.integrand * res_ucw(dst);
        color[ri] = make_float4(c.x, c.y, c.z, 1.f);
    }
}

__global__ void __launch_bounds__(128) k_sp_combine(uint32_t slot, SpatialCtx S, float4* __restrict__ color)
{
    sp_combine_body(slot, S, color, Blk{blockIdx.x, 8u});
}

__global__ void __launch_bounds__(128) kb_sp_combine(BatchQueue q, const SpatialColorArgs* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const SpatialColorArgs& a = args[inst];
        sp_combine_body(__ldg(q.slot + inst), a.S, a.color, batch_blk(q, inst, t));
    }
}


// ============================================================ MultiSplatting, wavefront form
// MultiScatterTemporalResampling.rt.slang:65-186 split like the ScatterBackup resampling: the shift
// mappings never use the generator's values, so the current sample's shift (k_ms_curr) and every
// splat's shift into its time partition (k_ms_splat, one thread per splat) run first and store their
// results; k_ms_combine replays the reference's resampling order and generator draws on them and
// rebuilds only the selected record.

// The current sample's scatter shift for its MIS weight (:96-117).
template <bool kEnv>
__global__ void __launch_bounds__(128, 8) k_ms_curr(uint32_t slot, MultiCtx M)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const bool useConf = C.useConfTemporal != 0;
    const uint32_t P = C.numTimePartitions;
    float timePartitions = C.camera.shutterSpeed / (float)P;
    Res cr = load_res(M.curr, ri);
    float currSampleMIS = 1.f;
    if (any_gt0(cr.integrand))
    {
        Recon crd = load_rec(M.currRec, ri);
        float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
        float fractionalTime = (crd.time - f_floor(crd.time / timePartitions) * timePartitions) / timePartitions;
        float shiftedTime = fractionalTime * C.camera.shutterSpeed;
        SampleGen dummy = {0, C.sgKind};
        Shifted sc = dev_scatter_shift<kEnv>(C, dummy, crd, shiftedTime + C.cm.artificialFrameTime, crd.firstHit, crd.lensSample, false);
        float sj = jac_scatter(sc, crd);
        float m2 = luminance(sc.radiance) * sj;
        m2 = f_isnan(m2) ? 0.f : m2;
        int spx = (int)f_floor(sc.fractionalPixel.x), spy = (int)f_floor(sc.fractionalPixel.y);
        if (valid_int(C, spx, spy)) m2 *= useConf ? load_confidence(M.prev, (uint32_t)spy * C.W + (uint32_t)spx) : 1.f;
        else m2 = 0.f;
        currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
    }
    M.currMIS[ri] = currSampleMIS;
}

// One splat of partition j (sorted position g = j * N + k) shifted to its partition's time (:124-160).
template <bool kEnv>
__global__ void __launch_bounds__(128, 8) k_ms_splat(uint32_t slot, MultiCtx M)
{
    const DevCtx& C = c_ctx[slot];
    const uint32_t N = C.W * C.H, P = C.numTimePartitions;
    uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P * N) return;
    const uint32_t j = g / N, k = g - j * N;
    if (k >= __ldg(&M.totals[j])) return;
    const bool useConf = C.useConfTemporal != 0;
    float timePartitions = C.camera.shutterSpeed / (float)P;
    const uint32_t si = __ldg(&M.sorted[g]), cell = __ldg(&M.sortedCell[g]);
    Res pr = load_res(M.prev, si);
    f3 prevPHat = mk3(0.f);
    float sj = 1.f, prevMIS = 0.f;
    f2 sub = pr.subPixel;
    if (any_gt0(pr.integrand))
    {
        Recon prd = load_rec(M.prevRec, si);
        float fractionalTime = prd.time / C.camera.shutterSpeed;
        float newTime = (fractionalTime + (float)j) * timePartitions;
        SampleGen dummy = {0, C.sgKind};
        Shifted sp = dev_scatter_shift<kEnv>(C, dummy, prd, newTime, prd.firstHit, prd.lensSample, false);
        store_shift(M.shift, g, sp);
        sj = jac_scatter(sp, prd);
        float m1 = luminance(sp.radiance) * sj * (useConf ? load_confidence(M.curr, cell) : 1.f);
        prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
        sj = f_isnan(m1) ? 1.f : sj;
        sub = sp.fractionalPixel - floor2(sp.fractionalPixel); // the record update's sub-pixel
        float m2 = luminance(pr.integrand) * (useConf ? pr.confidence : 1.f);
        prevMIS = ((m1 + m2) == 0.f) ? 0.f : m2 / (m1 + m2);
    }
    M.terms[g] = make_float4(prevPHat.x, prevPHat.y, prevPHat.z, sj);
    M.misSub[g] = make_float4(prevMIS, sub.x, sub.y, 0.f);
}

// The resampling of :90-186 in the reference's order (current sample, then partitions 0..P-1 and
// each cell's splats in sorted order) on the stored terms.
__global__ void __launch_bounds__(128) k_ms_combine(uint32_t slot, MultiCtx M, float4* __restrict__ color)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    const uint32_t N = C.W * C.H;
    uint32_t x = ri % C.W, y = ri / C.W;
    const bool useConf = C.useConfTemporal != 0;
    const uint32_t P = C.numTimePartitions;
    SampleGen sg = sg_create(x, y, pass_seed(C, 5), C.sgKind);
    Res dst = res_default();
    float jacobianScale = 1.f / (float)P;
    float timePartitions = C.camera.shutterSpeed / (float)P;
    Res cr = load_res_rw(M.curr, ri);
    bool selCurr = false, selZero = false;
    uint32_t selG = kInvalidIndex, selJ = 0;
    if (res_add_sample(dst, sg, M.currMIS[ri], cr.integrand, 1.f, cr)) selCurr = true;
    float newConfidence = dst.confidence;
    for (uint32_t j = 0; j < P; j++)
    {
        uint32_t n = __ldg(&M.counts[(size_t)j * N + ri]), off = __ldg(&M.offsets[(size_t)j * N + ri]);
        for (uint32_t i = 0; i < n; i++)
        {
            const uint32_t g = j * N + off + i;
            const uint32_t si = __ldg(&M.sorted[g]);
            Res pr = load_res(M.prev, si);
            const float4 t = __ldg(&M.terms[g]), m = __ldg(&M.misSub[g]);
            const bool live = any_gt0(pr.integrand);
            if (live) pr.subPixel = mk2(m.y, m.z);
            if (res_add_sample(dst, sg, m.x, mk3(t.x, t.y, t.z), t.w * jacobianScale, pr))
            {
                selCurr = false; selG = g; selJ = j; selZero = !live;
            }
        }
    }
    dst.confidence = bilinear_confidence(C, M.mvec, M.prev, x, y, newConfidence, useConf);
    store_res(M.curr, ri, dst);
    Recon dstR = recon_default();
    if (selCurr) dstR = load_rec_rw(M.currRec, ri);
    else if (selG != kInvalidIndex)
    {
        dstR = load_rec(M.prevRec, __ldg(&M.sorted[selG]));
        if (!selZero)
        {
            float fractionalTime = dstR.time / C.camera.shutterSpeed;
            float newTime = (fractionalTime + (float)selJ) * timePartitions;
            recon_update(dstR, load_shift(M.shift, selG));
            dstR.time = newTime;
        }
    }
    store_rec(M.currRec, ri, dstR);
    write_color(color, ri, dst);
}

} // namespace rs
