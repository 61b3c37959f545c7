// tb_reorder.cu -- reorder_particles! on the device
// (Tesserae.jl src/Parallel/gpu_block_strategy.jl:172-238, policy and score
// documented at src/Parallel/cpu_block_strategy.jl:221-269).
//
// The score is the reference's GPU estimator: the fraction of neighbouring
// particles in memory that share a (non-zero) block, over nassigned - nactive
// (1 when that is not positive). A reorder permutes every particle field
// through the partition's block-sorted permutation, permutes the block ids the
// same way and sets the permutation to the identity, so that the partition
// still describes the particles.
//
// Every kernel here reads the decision word on the device and returns at once
// when it is 0, so a fused step can apply the threshold policy without a host
// round trip. The permutation is a gather into a scratch array followed by a
// copy back into the caller's array (the caller's addresses do not change).
#include "tb_launch.cuh"

namespace tb {

namespace {

constexpr int RO_THREADS = 256;

// nassigned = offsets[nb]; nactive = number of non-empty blocks. Both come from
// the partition arrays themselves, so the partition may come from any binning.
__global__ void __launch_bounds__(RO_THREADS) reorder_score_kernel(const int* __restrict__ blockids, long long n,
                                                                   const int* __restrict__ counts, int nb,
                                                                   unsigned long long* __restrict__ acc) {
    unsigned long long same = 0, active = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p + 1 < n; p += stride) {
        const int a = blockids[p];
        same += (a != 0 && a == blockids[p + 1]);
    }
    for (long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += stride) active += counts[b] > 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        same += __shfl_down_sync(0xffffffffu, same, o);
        active += __shfl_down_sync(0xffffffffu, active, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (same) atomicAdd(acc + 0, same);
        if (active) atomicAdd(acc + 1, active);
    }
}

// decision[0] = 1 to reorder; decision[1] = 1 if a reorder was wanted but
// particles lie outside the mesh; score[0] = the contiguity score.
__global__ void reorder_decide_kernel(const unsigned long long* __restrict__ acc, const int* __restrict__ offsets,
                                      int nb, long long n, double threshold, int* __restrict__ decision,
                                      double* __restrict__ score, int* __restrict__ err) {
    const long long nassigned = offsets[nb];
    const long long maxsame = nassigned - (long long)acc[1];
    const double frac = maxsame <= 0 ? 1.0 : double(acc[0]) / double(maxsame);
    score[0] = frac;
    const bool want = threshold > 0.0 && (threshold >= 1.0 || frac < threshold) && n > 0;
    const bool all_in = nassigned == n;
    decision[0] = want && all_in;
    decision[1] = want && !all_in;
    if (want && !all_in && err) atomicOr(err, ERR_REORDER_OUTSIDE);
}

template <class E>
__global__ void __launch_bounds__(RO_THREADS) gather_kernel(const int* __restrict__ decision, long long n,
                                                            const int* __restrict__ perm, const E* __restrict__ src,
                                                            E* __restrict__ dst) {
    if (!decision[0]) return;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
        dst[j] = src[perm[j] - 1];
}

template <class E>
__global__ void __launch_bounds__(RO_THREADS) copy_kernel(const int* __restrict__ decision, long long n,
                                                          const E* __restrict__ src, E* __restrict__ dst) {
    if (!decision[0]) return;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
        dst[j] = src[j];
}

__global__ void __launch_bounds__(RO_THREADS) iota_kernel(const int* __restrict__ decision, long long n,
                                                          int* __restrict__ perm) {
    if (!decision[0]) return;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < n; j += (long long)gridDim.x * blockDim.x)
        perm[j] = int(j + 1);
}

}  // namespace

cudaError_t launch_reorder_score(const ReorderArgs& a, const LaunchCfg& cfg) {
    cudaError_t e = cudaMemsetAsync(a.acc, 0, 2 * sizeof(unsigned long long), cfg.stream);
    if (e != cudaSuccess) return e;
    const long long work = std::max<long long>(a.n, a.nblocks);
    const int grid = int(std::max<long long>(1, std::min<long long>((work + RO_THREADS - 1) / RO_THREADS,
                                                                    (long long)cfg.num_sms * 8)));
    KernelScope ks(cfg, "reorder_score");
    reorder_score_kernel<<<grid, RO_THREADS, 0, cfg.stream>>>(a.blockids, a.n, a.counts, a.nblocks, a.acc);
    reorder_decide_kernel<<<1, 1, 0, cfg.stream>>>(a.acc, a.offsets, a.nblocks, a.n, a.threshold, a.decision,
                                                   a.score, a.report_outside ? cfg.err : nullptr);
    *cfg.launches += 2;
    return cudaGetLastError();
}

cudaError_t launch_reorder_apply(const ReorderArgs& a, const ReorderField* fields, int nfields, const LaunchCfg& cfg) {
    if (a.n <= 0) return cudaSuccess;
    const int grid = int(std::max<long long>(1, std::min<long long>((a.n + RO_THREADS - 1) / RO_THREADS,
                                                                    (long long)cfg.num_sms * 16)));
    KernelScope ks(cfg, "reorder");
    for (int i = 0; i < nfields; ++i) {
        const ReorderField& f = fields[i];
        if (f.elem == 8) {
            gather_kernel<unsigned long long><<<grid, RO_THREADS, 0, cfg.stream>>>(
                a.decision, a.n, a.perm, static_cast<const unsigned long long*>(f.ptr),
                static_cast<unsigned long long*>(a.scratch));
            copy_kernel<unsigned long long><<<grid, RO_THREADS, 0, cfg.stream>>>(
                a.decision, a.n, static_cast<const unsigned long long*>(a.scratch),
                static_cast<unsigned long long*>(f.ptr));
        } else {
            gather_kernel<unsigned><<<grid, RO_THREADS, 0, cfg.stream>>>(a.decision, a.n, a.perm,
                                                                        static_cast<const unsigned*>(f.ptr),
                                                                        static_cast<unsigned*>(a.scratch));
            copy_kernel<unsigned><<<grid, RO_THREADS, 0, cfg.stream>>>(a.decision, a.n,
                                                                      static_cast<const unsigned*>(a.scratch),
                                                                      static_cast<unsigned*>(f.ptr));
        }
        *cfg.launches += 2;
    }
    // block ids follow the particles; the permutation becomes the identity
    gather_kernel<int><<<grid, RO_THREADS, 0, cfg.stream>>>(a.decision, a.n, a.perm, a.blockids,
                                                           static_cast<int*>(a.scratch));
    copy_kernel<int><<<grid, RO_THREADS, 0, cfg.stream>>>(a.decision, a.n, static_cast<const int*>(a.scratch),
                                                         a.blockids);
    iota_kernel<<<grid, RO_THREADS, 0, cfg.stream>>>(a.decision, a.n, a.perm);
    *cfg.launches += 3;
    return cudaGetLastError();
}

}  // namespace tb
