// Batched sweep: the plan and streaming kernels and the FP64 level kernel.
// Compiled with -fmad=false, like device_ops.cu, so a member's FP64 sweep
// and its streaming passes round exactly as in the single-instance path.
#include "batch_kernels.cuh"

namespace tycho {

namespace {

// Grid-stride loop over the active members' phi chunks: fn(slot, first
// element, end element, chunk index).
template <typename Fn>
__device__ __forceinline__ void for_each_chunk(const BatchSlot *__restrict__ slots, const BatchPlan &pl, Fn fn)
{
    const uint32_t n_act = *pl.n_act;
    const uint32_t total = pl.chunk_prefix[n_act];
    for (uint32_t b = blockIdx.x; b < total; b += gridDim.x) {
        const uint32_t k = upper_index(n_act, b, [&](uint32_t m) { return pl.chunk_prefix[m]; });
        const BatchSlot &s = slots[pl.act[k]];
        const uint64_t n = s.nc * 4 * s.G;
        const uint64_t i0 = (uint64_t)(b - pl.chunk_prefix[k]) * kBatchChunk;
        const uint64_t i1 = i0 + kBatchChunk < n ? i0 + kBatchChunk : n;
        fn(s, i0, i1, b);
    }
}

__global__ void __launch_bounds__(256) batch_accept_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl)
{
    for_each_chunk(slots, pl, [&](const BatchSlot &s, uint64_t i0, uint64_t i1, uint32_t) {
        if (!s.accept) return;
        for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) s.phi[i] = s.phi[i] + s.vec_d[i];
    });
}

// One thread per (cell, group) of the chunk when chunks hold whole cells
// (4 G divides the chunk size), as in the single-instance scatter; else one
// per element.  Bit-identical either way.
__global__ void __launch_bounds__(256) batch_scatter_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl)
{
    for_each_chunk(slots, pl, [&](const BatchSlot &s, uint64_t i0, uint64_t i1, uint32_t) {
        const uint32_t row = 4u * s.G;
        if (kBatchChunk % row == 0) {
            const uint64_t c0 = i0 / row;
            const uint32_t pairs = (uint32_t)((i1 - i0) / 4);
            for (uint32_t q = threadIdx.x; q < pairs; q += blockDim.x) {
                const uint32_t dc = q / s.G, g = q - dc * s.G;
                double v[4];
                scatter_cell_group(s.phi_in, s.q_fixed, s.sigma_s, s.scat, c0 + dc, g, s.G, v);
                const uint64_t base = (c0 + dc) * row + g;
#pragma unroll
                for (int k = 0; k < 4; ++k) s.iso[base + k * s.G] = v[k];
                if (s.iso32) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) s.iso32[base + k * s.G] = (float)v[k];
                }
            }
            return;
        }
        for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const double v = scatter_elem(s.phi_in, s.q_fixed, s.sigma_s, s.scat, i, s.G);
            s.iso[i] = v;
            if (s.iso32) s.iso32[i] = (float)v;
        }
    });
}

template <typename Real>
__global__ void __launch_bounds__(256) batch_psi_to_phi_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl)
{
    for_each_chunk(slots, pl, [&](const BatchSlot &s, uint64_t i0, uint64_t i1, uint32_t) {
        // from 8 groups on one element per thread (a warp's elements share
        // a 128-byte line per angle), else four (chunks and rows are
        // multiples of 4)
        const Real *psi = (const Real *)s.psi;
        if (s.G >= 8) {
            for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x)
                s.phi_out[i] = psi_to_phi_elem8(psi, s.w, i, s.A, s.G);
            return;
        }
        for (uint64_t i = i0 + 4 * threadIdx.x; i < i1; i += 4 * blockDim.x) {
            double v[4];
            psi_to_phi_quad(psi, s.w, i, s.A, s.G, v);
            reinterpret_cast<double2 *>(s.phi_out + i)[0] = make_double2(v[0], v[1]);
            reinterpret_cast<double2 *>(s.phi_out + i)[1] = make_double2(v[2], v[3]);
        }
    });
}

// Per element of an active member, by its op:
//   kOpSI     d += |out - in|, m += |out|                   (out = phi_out, in = phi_in)
//   kOpOuter  r = out - phi (into vec_r and vec_d); d += |r|, m += |out|
//   kOpInner  dn = r + out; d += |dn - delta|, m += |dn|; delta = dn
// with one (d, m) partial per chunk in a fixed order.
__global__ void __launch_bounds__(256) batch_post_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl)
{
    __shared__ double sh[8][2];
    for_each_chunk(slots, pl, [&](const BatchSlot &s, uint64_t i0, uint64_t i1, uint32_t b) {
        double d = 0.0, m = 0.0;
        for (uint64_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
            const double out = s.phi_out[i];
            if (s.op == kOpSI) {
                d += fabs(out - s.phi_in[i]);
                m += fabs(out);
            } else if (s.op == kOpOuter) {
                const double r = out - s.phi[i];
                s.vec_r[i] = r;
                s.vec_d[i] = r;
                d += fabs(r);
                m += fabs(out);
            } else {
                const double dn = s.vec_r[i] + out;
                d += fabs(dn - s.vec_d[i]);
                m += fabs(dn);
                s.vec_d[i] = dn;
            }
        }
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        d = warp_sum(d);
        m = warp_sum(m);
        if (lane == 0) { sh[warp][0] = d; sh[warp][1] = m; }
        __syncthreads();
        if (threadIdx.x < 2) {
            double t = 0.0;
            for (int q = 0; q < 8; ++q) t += sh[q][threadIdx.x];
            pl.partials[(size_t)b * 2 + threadIdx.x] = t;
        }
        __syncthreads();
    });
}

// One warp per active member: its chunk partials in chunk order (lane l
// takes chunks l, l + 32, ...; then a fixed shuffle tree).
__global__ void __launch_bounds__(256) batch_finish_kernel(const BatchSlot *__restrict__ slots, BatchPlan pl)
{
    const uint32_t n_act = *pl.n_act;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k = blockIdx.x * 8u + (threadIdx.x >> 5); k < n_act; k += gridDim.x * 8u) {
        const uint32_t c0 = pl.chunk_prefix[k], c1 = pl.chunk_prefix[k + 1];
        double d = 0.0, m = 0.0;
        for (uint32_t c = c0 + lane; c < c1; c += 32) {
            d += pl.partials[(size_t)c * 2];
            m += pl.partials[(size_t)c * 2 + 1];
        }
        d = warp_sum(d);
        m = warp_sum(m);
        if (lane == 0) {
            const uint32_t j = pl.act[k];
            pl.norms[(size_t)j * 2] = d;
            pl.norms[(size_t)j * 2 + 1] = m;
        }
    }
    (void)slots;
}

cudaError_t level_launch(const void *fn, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                         const BatchCuts &cut, cudaStream_t s)
{
    const unsigned grid = cut.c[kBatchClasses];
    if (grid == 0) return cudaSuccess;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&slots, (void *)&pl, (void *)&level, (void *)&cut};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace

cudaError_t batch_level_launch(const void *fn, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                               const BatchCuts &cut, cudaStream_t s)
{
    return level_launch(fn, slots, pl, level, cut, s);
}

template <>
cudaError_t launch_batch_level<double>(int ipw, const BatchSlot *slots, const BatchPlan &pl, uint32_t level,
                                       const BatchCuts &cut, bool any_solver, cudaStream_t s)
{
    const void *fn = ipw == 0    ? (any_solver ? (const void *)batch_direct_level_kernel<double, true>
                                               : (const void *)batch_direct_level_kernel<double, false, 4>)
                     : ipw == 8  ? (const void *)batch_level_kernel<double, 8>
                     : ipw == 16 ? (const void *)batch_level_kernel<double, 16>
                     : ipw == 32 ? (const void *)batch_level_kernel<double, 32>
                                 : nullptr;
    if (!fn) return cudaErrorInvalidValue;
    return level_launch(fn, slots, pl, level, cut, s);
}

template <>
cudaError_t launch_batch_persist<double>(const BatchSlot *slots, const BatchPlan &pl, const BatchPersistArgs &a,
                                         bool any_solver, cudaStream_t s)
{
    return any_solver ? batch_persist_launch<double, true, 1>(slots, pl, a, s)
                      : batch_persist_launch<double, false, 4>(slots, pl, a, s);
}

cudaError_t launch_batch_plan(int ipw, const BatchSlot *slots, uint32_t n_slots, uint32_t max_levels,
                              uint32_t rec_bytes, const BatchPlan &pl, cudaStream_t s)
{
    const dim3 grid(max_levels + 1), block(kBatchPlanThreads);
    switch (ipw) {
    case 0: batch_plan_kernel<0><<<grid, block, 0, s>>>(slots, n_slots, max_levels, rec_bytes, pl); break;
    case 8: batch_plan_kernel<8><<<grid, block, 0, s>>>(slots, n_slots, max_levels, rec_bytes, pl); break;
    case 16: batch_plan_kernel<16><<<grid, block, 0, s>>>(slots, n_slots, max_levels, rec_bytes, pl); break;
    case 32: batch_plan_kernel<32><<<grid, block, 0, s>>>(slots, n_slots, max_levels, rec_bytes, pl); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_batch_accept(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s)
{
    batch_accept_kernel<<<grid, 256, 0, s>>>(slots, pl);
    return cudaGetLastError();
}

cudaError_t launch_batch_scatter(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s)
{
    batch_scatter_kernel<<<grid, 256, 0, s>>>(slots, pl);
    return cudaGetLastError();
}

cudaError_t launch_batch_psi_to_phi(bool fp32, const BatchSlot *slots, const BatchPlan &pl, unsigned grid,
                                    cudaStream_t s)
{
    if (fp32) batch_psi_to_phi_kernel<float><<<grid, 256, 0, s>>>(slots, pl);
    else batch_psi_to_phi_kernel<double><<<grid, 256, 0, s>>>(slots, pl);
    return cudaGetLastError();
}

cudaError_t launch_batch_post(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s)
{
    batch_post_kernel<<<grid, 256, 0, s>>>(slots, pl);
    return cudaGetLastError();
}

cudaError_t launch_batch_finish(const BatchSlot *slots, const BatchPlan &pl, unsigned grid, cudaStream_t s)
{
    batch_finish_kernel<<<grid, 256, 0, s>>>(slots, pl);
    return cudaGetLastError();
}

}  // namespace tycho
