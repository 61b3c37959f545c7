// tb_bin.cu -- particle binning into grid blocks: the device counterpart of
// update!(::GPUBlockStrategy, x) (Tesserae.jl src/Parallel/gpu_block_strategy.jl:142-166),
// producing the block order of the reference CPU strategy bit for bit: block id
// ascending, particle id ascending inside a block (cpu_block_strategy.jl:174-190).
//
//   count    one thread per particle: findblock, warp-aggregated count atomics
//   scan     3 launches over packed (count | nonempty << 32) 64-bit sums: tile
//            reduce, single-CTA spine, tile rescan writing offsets, cursors,
//            the compacted block list and the totals [nactive, nassigned]
//   scatter  a warp takes 4 chunks of 32 ids and reserves one run per (chunk,
//            distinct block) with a single atomic, writing the particles in lane order
//   fixup    one warp per non-empty block: the block's segment is a set of runs,
//            one per scatter warp (32 consecutive particle ids), each ascending;
//            the runs are ranked by warp id and copied in order. Blocks of more
//            than 64 runs are sorted by a second kernel (one CTA per block,
//            bitonic in shared memory, or in a global scratch region for
//            segments above 2048 runs).
// The result is deterministic regardless of atomic order.
#include "tb_launch.cuh"

namespace tb {

namespace {

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <int D, class T>
__global__ void __launch_bounds__(256) bin_count_kernel(DMesh<D, T> M, const T* __restrict__ x0,
                                                        const T* __restrict__ x1, const T* __restrict__ x2,
                                                        long long n, int* __restrict__ blockids,
                                                        int* __restrict__ counts) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int b = -1;
    if (p < n) {
        T x[3];
        x[0] = x0[p];
        x[1] = x1[p];
        if constexpr (D == 3) x[2] = x2[p];
        b = findblock<D, T>(M, x);
        blockids[p] = b;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int leader = __ffs(peers) - 1;
    if (b > 0 && int(threadIdx.x & 31) == leader) atomicAdd(&counts[b - 1], __popc(peers));
}

__device__ __forceinline__ unsigned long long pack_count(int c) {
    return (unsigned long long)(unsigned)c | ((unsigned long long)(c != 0) << 32);
}

// Inclusive block scan of one 64-bit value per thread (blockDim = 256).
__device__ __forceinline__ unsigned long long block_incl_scan(unsigned long long v, unsigned long long* warp_tot,
                                                              unsigned long long& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[wid] = v;
    __syncthreads();
    if (wid == 0) {
        unsigned long long w = lane < nw ? warp_tot[lane] : 0ull;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    total = warp_tot[nw - 1];
    unsigned long long r = v + (wid > 0 ? warp_tot[wid - 1] : 0ull);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) scan_reduce_kernel(const int* __restrict__ counts, int nb,
                                                          unsigned long long* __restrict__ partials) {
    __shared__ unsigned long long wt[8];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
    unsigned long long s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (base + k < nb) s += pack_count(counts[base + k]);
    unsigned long long total;
    block_incl_scan(s, wt, total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Exclusive scan of the tile partials in place (one CTA).
__global__ void __launch_bounds__(256) scan_spine_kernel(unsigned long long* partials, int ntiles) {
    __shared__ unsigned long long wt[8];
    unsigned long long carry = 0;
    for (int c = 0; c < ntiles; c += 256) {
        const int i = c + threadIdx.x;
        unsigned long long v = i < ntiles ? partials[i] : 0ull;
        unsigned long long total;
        unsigned long long incl = block_incl_scan(v, wt, total);
        if (i < ntiles) partials[i] = carry + incl - v;
        carry += total;
    }
}

__global__ void __launch_bounds__(256) scan_finalize_kernel(const int* __restrict__ counts, int nb,
                                                            const unsigned long long* __restrict__ partials,
                                                            int* __restrict__ offsets, int* __restrict__ cursors,
                                                            int* __restrict__ blocklist, int* __restrict__ totals) {
    __shared__ unsigned long long wt[8];
    const int base = blockIdx.x * SCAN_TILE + threadIdx.x * 4;
    int c[4];
    unsigned long long s = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        c[k] = (base + k < nb) ? counts[base + k] : 0;
        s += pack_count(c[k]);
    }
    unsigned long long total;
    unsigned long long incl = block_incl_scan(s, wt, total);
    unsigned long long run = partials[blockIdx.x] + incl - s;  // exclusive prefix of this thread
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int b = base + k;
        if (b < nb) {
            const int start = int(run & 0xffffffffull);
            offsets[b] = start;
            cursors[b] = start;
            if (c[k] != 0) blocklist[int(run >> 32)] = b + 1;
            run += pack_count(c[k]);
            if (b == nb - 1) {
                offsets[nb] = int(run & 0xffffffffull);
                totals[0] = int(run >> 32);
                totals[1] = int(run & 0xffffffffull);
            }
        }
    }
}

// Each warp scatters SCAT_IT chunks of 32 consecutive ids: all their block ids
// are loaded, and all their run reservations issued, before any is waited for
// (one round trip each instead of one per chunk). A chunk still reserves one
// run per block, so the runs the fix-up orders are those of one warp per chunk.
constexpr int SCAT_IT = 4;
__global__ void __launch_bounds__(256) bin_scatter_kernel(const int* __restrict__ blockids, long long n,
                                                          int* __restrict__ cursors, int* __restrict__ perm_tmp) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const long long c0 = (((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5) * (32ll * SCAT_IT);
    int b[SCAT_IT];
#pragma unroll
    for (int u = 0; u < SCAT_IT; ++u) {
        const long long p = c0 + 32 * u + lane;
        b[u] = p < n ? blockids[p] : -1;
    }
    unsigned peers[SCAT_IT];
    int base[SCAT_IT];
#pragma unroll
    for (int u = 0; u < SCAT_IT; ++u) {
        peers[u] = __match_any_sync(full, b[u]);
        base[u] = 0;
        if (b[u] > 0 && lane == __ffs(peers[u]) - 1) base[u] = atomicAdd(&cursors[b[u] - 1], __popc(peers[u]));
    }
#pragma unroll
    for (int u = 0; u < SCAT_IT; ++u) {
        const int bb = __shfl_sync(full, base[u], __ffs(peers[u]) - 1);
        if (b[u] > 0) perm_tmp[bb + __popc(peers[u] & lanemask_lt())] = int(c0 + 32 * u + lane);
    }
}

constexpr int FIX_THREADS = 256;
constexpr int FIX_SMEM_KEYS = 2048;

__device__ __forceinline__ int next_pow2(int v) {
    int k = 1;
    while (k < v) k <<= 1;
    return k;
}

// Exclusive scan of one int per thread over the CTA (blockDim = FIX_THREADS);
// `total` gets the sum. Two barriers; `wsum` holds the warp sums.
__device__ __forceinline__ int fix_excl_scan(int v, int* wsum, int& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    int wprefix = 0;
    total = 0;
#pragma unroll
    for (int q = 0; q < FIX_THREADS / 32; ++q) {
        const int w = wsum[q];
        wprefix += q < wid ? w : 0;
        total += w;
    }
    __syncthreads();
    return wprefix + incl - v;
}

// Blocks of more than FIXW_RUNS runs, one CTA per block. Runs are found in
// segment order, their keys (scatter warp id << 32 | run index) bitonic-sorted,
// the output start of each run is the prefix sum of the run lengths in sorted
// order, and the segment is copied element-parallel (each element to its run's
// place), all in shared memory when the padded key count fits; above that
// (more than FIX_SMEM_KEYS runs) the keys are sorted in the block's own region
// [2s, 2s + 2n) of the global scratch (next_pow2(k) <= 2n, segments disjoint)
// and each thread copies whole runs.
__global__ void __launch_bounds__(FIX_THREADS) bin_fixup_kernel(const int* __restrict__ totals,
                                                                const int* __restrict__ blocklist,
                                                                const int* __restrict__ offsets,
                                                                const int* __restrict__ counts,
                                                                const int* __restrict__ S, int* __restrict__ perm,
                                                                unsigned long long* __restrict__ gscratch) {
    __shared__ unsigned long long sbuf[FIX_SMEM_KEYS];
    __shared__ int hpos[FIX_SMEM_KEYS + 1];  // run starts, segment order
    __shared__ int hout[FIX_SMEM_KEYS];      // output start of each run, segment order
    __shared__ int kcount;
    __shared__ int wsum[FIX_THREADS / 32];
    const int nactive = totals[0];
    const int tid = threadIdx.x;
    auto is_head = [](const int* seg, int j, int v) { return j == 0 || (seg[j - 1] >> 5) != (v >> 5); };
    for (int bi = blockIdx.x; bi < nactive; bi += gridDim.x) {
        const int b = blocklist[bi] - 1;
        const int s = offsets[b];
        const int n = counts[b];
        const int* seg = S + s;
        int* out = perm + s;
        // Run heads: the first element, and every element whose warp id differs
        // from its predecessor's.
        int myheads = 0;
        for (int j = tid; j < n; j += FIX_THREADS) myheads += is_head(seg, j, seg[j]);
        int k;
        fix_excl_scan(myheads, wsum, k);
        const int K = next_pow2(k);
        if (K <= FIX_SMEM_KEYS) {
            // 1. heads in segment order: positions and keys
            int rbase = 0;
            for (int j0 = 0; j0 < n; j0 += FIX_THREADS) {
                const int j = j0 + tid;
                const int v = j < n ? seg[j] : 0;
                const int h = (j < n && is_head(seg, j, v)) ? 1 : 0;
                int tot;
                const int r = rbase + fix_excl_scan(h, wsum, tot);
                if (h) {
                    hpos[r] = j;
                    sbuf[r] = ((unsigned long long)(unsigned)(v >> 5) << 32) | (unsigned)r;
                }
                rbase += tot;
            }
            if (tid == 0) hpos[k] = n;
            for (int t = k + tid; t < K; t += FIX_THREADS) sbuf[t] = ~0ull;
            __syncthreads();
            // 2. bitonic sort of the K keys (ascending)
            for (int size = 2; size <= K; size <<= 1) {
                for (int stride = size >> 1; stride > 0; stride >>= 1) {
                    for (int i = tid; i < (K >> 1); i += FIX_THREADS) {
                        const int lo = (i / stride) * 2 * stride + (i % stride);
                        const int hi = lo + stride;
                        const bool asc = (lo & size) == 0;
                        const unsigned long long a = sbuf[lo], c = sbuf[hi];
                        if ((a > c) == asc) {
                            sbuf[lo] = c;
                            sbuf[hi] = a;
                        }
                    }
                    __syncthreads();
                }
            }
            // 3. output start of each run: lengths summed in sorted order
            int obase = 0;
            for (int i0 = 0; i0 < k; i0 += FIX_THREADS) {
                const int i = i0 + tid;
                int r = 0, len = 0;
                if (i < k) {
                    r = int(sbuf[i] & 0xffffffffull);
                    len = hpos[r + 1] - hpos[r];
                }
                int tot;
                const int st = obase + fix_excl_scan(len, wsum, tot);
                if (i < k) hout[r] = st;
                obase += tot;
            }
            __syncthreads();
            // 4. element-parallel copy: an element's run is the number of heads at
            //    or before it, minus one
            rbase = 0;
            for (int j0 = 0; j0 < n; j0 += FIX_THREADS) {
                const int j = j0 + tid;
                const int v = j < n ? seg[j] : 0;
                const int h = (j < n && is_head(seg, j, v)) ? 1 : 0;
                int tot;
                const int r = rbase + fix_excl_scan(h, wsum, tot) + h - 1;
                if (j < n) out[hout[r] + (j - hpos[r])] = v + 1;
                rbase += tot;
            }
            __syncthreads();
            continue;
        }
        unsigned long long* buf = gscratch + 2ll * s;
        if (tid == 0) kcount = 0;
        __syncthreads();
        for (int j = tid; j < n; j += FIX_THREADS) {
            const int v = seg[j];
            if (is_head(seg, j, v)) {
                const int idx = atomicAdd(&kcount, 1);
                buf[idx] = ((unsigned long long)(unsigned)(v >> 5) << 32) | (unsigned)j;
            }
        }
        __syncthreads();
        for (int t = k + tid; t < K; t += FIX_THREADS) buf[t] = ~0ull;
        __syncthreads();
        // Bitonic sort of the K keys (ascending).
        for (int size = 2; size <= K; size <<= 1) {
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int i = tid; i < (K >> 1); i += FIX_THREADS) {
                    const int lo = (i / stride) * 2 * stride + (i % stride);
                    const int hi = lo + stride;
                    const bool asc = (lo & size) == 0;
                    const unsigned long long a = buf[lo], c = buf[hi];
                    if ((a > c) == asc) {
                        buf[lo] = c;
                        buf[hi] = a;
                    }
                }
                __syncthreads();
            }
        }
        // Copy the runs in sorted order; each run is at most 32 long.
        int base = 0;
        for (int c0 = 0; c0 < k; c0 += FIX_THREADS) {
            const int r = c0 + tid;
            int len = 0, j0 = 0;
            if (r < k) {
                const unsigned long long e = buf[r];
                j0 = int(e & 0xffffffffull);
                const int w = int(e >> 32);
                len = 1;
                while (j0 + len < n && (seg[j0 + len] >> 5) == w) ++len;
            }
            int total;
            const int excl = base + fix_excl_scan(len, wsum, total);
            for (int t = 0; t < len; ++t) out[excl + t] = seg[j0 + t] + 1;
            base += total;
        }
        __syncthreads();
    }
}

// One warp per non-empty block: the block's segment of the scattered ids is a
// concatenation of runs, one per scatter warp that held particles of the block,
// each ascending and contiguous, and no two runs of a segment share a warp id.
// The warp finds the run heads with ballots, ranks the runs by warp id (every
// run against every run, at most FIXW_RUNS of them) and copies the segment
// element-parallel, each element to its run's place. A block with more runs is appended to an
// overflow list that bin_fixup_kernel then sorts.
constexpr int FIXW_RUNS = 64;
constexpr int FIXW_U = 8;  // chunks of 32 ids loaded together
constexpr int FIXW_THREADS = 256;

__global__ void __launch_bounds__(FIXW_THREADS) bin_fixup_warp_kernel(const int* __restrict__ totals,
                                                                      const int* __restrict__ blocklist,
                                                                      const int* __restrict__ offsets,
                                                                      const int* __restrict__ counts,
                                                                      const int* __restrict__ S,
                                                                      int* __restrict__ perm,
                                                                      int* __restrict__ overflow,
                                                                      unsigned long long* __restrict__ noverflow) {
    constexpr int NWARP = FIXW_THREADS / 32;
    __shared__ int hpos[NWARP][FIXW_RUNS + 1];
    __shared__ int hkey[NWARP][FIXW_RUNS];
    __shared__ int hout[NWARP][FIXW_RUNS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int nactive = totals[0];
    const unsigned full = 0xffffffffu;
    const unsigned below = (1u << lane) - 1u;
    for (int bi = blockIdx.x * NWARP + w; bi < nactive; bi += gridDim.x * NWARP) {
        const int b = blocklist[bi] - 1;
        const int s = offsets[b], n = counts[b];
        const int* seg = S + s;
        int* out = perm + s;
        int nruns = 0;
        // A run is at most 32 long, so a longer segment has too many runs: hand it
        // over without walking it (one warp reading thousands of ids serially was
        // most of the fix-up time of crowded scenes), and stop walking at the
        // first run past the limit.
        if (n > FIXW_RUNS * 32) nruns = FIXW_RUNS + 1;
        // The segment is read FIXW_U chunks of 32 at a time, all loads of a batch
        // issued before any is used; the predecessor of a chunk's first element
        // is lane 31 of the chunk before.
        int last = -1;
        for (int J0 = 0; J0 < n && nruns <= FIXW_RUNS; J0 += 32 * FIXW_U) {
            int vv[FIXW_U];
#pragma unroll
            for (int u = 0; u < FIXW_U; ++u) {
                const int j = J0 + 32 * u + lane;
                vv[u] = j < n ? seg[j] : 0;
            }
#pragma unroll
            for (int u = 0; u < FIXW_U; ++u) {
                const int j0 = J0 + 32 * u;
                if (j0 >= n) break;
                const int j = j0 + lane, v = vv[u];
                int prev = __shfl_up_sync(full, v, 1);
                if (lane == 0) prev = last;
                last = __shfl_sync(full, v, 31);
                const bool head = j < n && (j == 0 || (prev >> 5) != (v >> 5));
                const unsigned hm = __ballot_sync(full, head);
                const int idx = nruns + __popc(hm & below);
                if (head && idx < FIXW_RUNS) {
                    hpos[w][idx] = j;
                    hkey[w][idx] = v >> 5;
                }
                nruns += __popc(hm);
            }
        }
        if (nruns > FIXW_RUNS) {
            if (lane == 0) overflow[atomicAdd(noverflow, 1ull)] = b + 1;
            __syncwarp();
            continue;
        }
        if (lane == 0) hpos[w][nruns] = n;
        __syncwarp();
        // output start of each run: total length of the runs with a smaller warp id
        for (int r = lane; r < nruns; r += 32) {
            const int key = hkey[w][r];
            int start = 0;
            for (int q = 0; q < nruns; ++q)
                if (hkey[w][q] < key) start += hpos[w][q + 1] - hpos[w][q];
            hout[w][r] = start;
        }
        __syncwarp();
        // copy element-parallel: the run of element j is the number of heads at
        // or before j, minus one
        int rbase = 0;
        last = -1;
        for (int J0 = 0; J0 < n; J0 += 32 * FIXW_U) {
            int vv[FIXW_U];
#pragma unroll
            for (int u = 0; u < FIXW_U; ++u) {
                const int j = J0 + 32 * u + lane;
                vv[u] = j < n ? seg[j] : 0;
            }
#pragma unroll
            for (int u = 0; u < FIXW_U; ++u) {
                const int j0 = J0 + 32 * u;
                if (j0 >= n) break;
                const int j = j0 + lane, v = vv[u];
                int prev = __shfl_up_sync(full, v, 1);
                if (lane == 0) prev = last;
                last = __shfl_sync(full, v, 31);
                const bool head = j < n && (j == 0 || (prev >> 5) != (v >> 5));
                const unsigned hm = __ballot_sync(full, head);
                const int r = rbase + __popc(hm & (below | (1u << lane))) - 1;
                if (j < n) out[hout[w][r] + (j - hpos[w][r])] = v + 1;
                rbase += __popc(hm);
            }
        }
        __syncwarp();
    }
}

inline unsigned grid_for(long long n, int threads) { return unsigned((n + threads - 1) / threads); }

// ---- sparse grid numbering ----------------------------------------------
// act[B] = 1 for every node block B within one block per axis of a block that
// holds particles (act zeroed before). Several threads may store the same 1.
template <int D>
__global__ void __launch_bounds__(128) sparse_mark_kernel(const int* __restrict__ totals,
                                                          const int* __restrict__ blocklist, int3 nb,
                                                          int* __restrict__ act) {
    const int nactive = totals[0];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nactive; i += gridDim.x * blockDim.x) {
        const int b = blocklist[i] - 1;
        const int bx = b % nb.x, by = (b / nb.x) % nb.y, bz = (D == 3) ? b / (nb.x * nb.y) : 0;
        for (int dz = (D == 3 ? -1 : 0); dz <= (D == 3 ? 1 : 0); ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = bx + dx, y = by + dy, z = bz + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= nb.x || y >= nb.y || (D == 3 && z >= nb.z)) continue;
                    act[x + nb.x * (y + nb.y * z)] = 1;
                }
    }
}

// bnum[B] = (rank of B among the active blocks) + 1, or 0; the count to nact[0].
__global__ void __launch_bounds__(256) sparse_number_kernel(const int* __restrict__ act,
                                                            const int* __restrict__ offsets, int nb,
                                                            const int* __restrict__ totals, int* __restrict__ bnum,
                                                            int* __restrict__ nact) {
    for (int B = blockIdx.x * blockDim.x + threadIdx.x; B < nb; B += gridDim.x * blockDim.x) {
        bnum[B] = act[B] ? offsets[B] + 1 : 0;
        if (B == 0) nact[0] = totals[0];
    }
}

}  // namespace

cudaError_t launch_sparsity(int dim, const int* nbv, int nblocks, const BinBuffers& b, const SparseScratch& sc,
                            int* bnum, int* blist, int* nact, const LaunchCfg& cfg) {
    cudaError_t e = cudaMemsetAsync(sc.act, 0, sizeof(int) * size_t(nblocks), cfg.stream);
    if (e != cudaSuccess) return e;
    KernelScope ks(cfg, "sparsity");
    const int3 nb = make_int3(nbv[0], nbv[1], nbv[2]);
    const int mgrid = std::max(1, std::min((nblocks + 127) / 128, cfg.num_sms * 8));
    if (dim == 3) sparse_mark_kernel<3><<<mgrid, 128, 0, cfg.stream>>>(b.totals, b.blocklist, nb, sc.act);
    else sparse_mark_kernel<2><<<mgrid, 128, 0, cfg.stream>>>(b.totals, b.blocklist, nb, sc.act);
    // the binning's scan over the activity: offsets = ranks, blocklist = the active list
    const int nt = scan_tiles(nblocks);
    scan_reduce_kernel<<<nt, 256, 0, cfg.stream>>>(sc.act, nblocks, sc.partials);
    scan_spine_kernel<<<1, 256, 0, cfg.stream>>>(sc.partials, nt);
    scan_finalize_kernel<<<nt, 256, 0, cfg.stream>>>(sc.act, nblocks, sc.partials, sc.offsets, sc.cursors, blist,
                                                     sc.totals);
    sparse_number_kernel<<<std::max(1, std::min((nblocks + 255) / 256, cfg.num_sms * 8)), 256, 0, cfg.stream>>>(
        sc.act, sc.offsets, nblocks, sc.totals, bnum, nact);
    *cfg.launches += 5;
    return cudaGetLastError();
}

template <int D, class T>
cudaError_t launch_bin_count(const DMesh<D, T>& M, const T* const* x, long long n, const BinBuffers& b,
                             const LaunchCfg& cfg) {
    cudaError_t e = cudaMemsetAsync(b.counts, 0, sizeof(int) * size_t(M.nblocks), cfg.stream);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        KernelScope ks(cfg, "bin_count");
        bin_count_kernel<D, T><<<grid_for(n, 256), 256, 0, cfg.stream>>>(M, x[0], x[1], D == 3 ? x[2] : x[1], n,
                                                                         b.blockids, b.counts);
        ++*cfg.launches;
    }
    return cudaGetLastError();
}

cudaError_t launch_bin_rest(int nb, long long n, const BinBuffers& b, const LaunchCfg& cfg) {
    const int nt = scan_tiles(nb);
    {
        KernelScope ks(cfg, "bin_scan");
        scan_reduce_kernel<<<nt, 256, 0, cfg.stream>>>(b.counts, nb, b.partials);
        scan_spine_kernel<<<1, 256, 0, cfg.stream>>>(b.partials, nt);
        scan_finalize_kernel<<<nt, 256, 0, cfg.stream>>>(b.counts, nb, b.partials, b.offsets, b.cursors, b.blocklist,
                                                         b.totals);
    }
    *cfg.launches += 3;
    if (n > 0) {
        {
            KernelScope ks(cfg, "bin_scatter");
            bin_scatter_kernel<<<grid_for(n, 256 * SCAT_IT), 256, 0, cfg.stream>>>(b.blockids, n, b.cursors,
                                                                                  b.perm_tmp);
        }
        // Blocks of more than FIXW_RUNS runs go to an overflow list kept in the
        // cursor array (free once the scatter is done), its length in partials[0].
        cudaError_t e = cudaMemsetAsync(b.partials, 0, sizeof(unsigned long long), cfg.stream);
        if (e != cudaSuccess) return e;
        KernelScope ks(cfg, "bin_fixup");
        const int wgrid = std::max(1, std::min((nb + FIXW_THREADS / 32 - 1) / (FIXW_THREADS / 32), cfg.num_sms * 8));
        bin_fixup_warp_kernel<<<wgrid, FIXW_THREADS, 0, cfg.stream>>>(b.totals, b.blocklist, b.offsets, b.counts,
                                                                      b.perm_tmp, b.perm, b.cursors, b.partials);
        const int grid = std::min(nb, cfg.num_sms * 16);
        bin_fixup_kernel<<<grid, FIX_THREADS, 0, cfg.stream>>>(reinterpret_cast<const int*>(b.partials), b.cursors,
                                                               b.offsets, b.counts, b.perm_tmp, b.perm,
                                                               b.sort_scratch);
        *cfg.launches += 3;
    }
    return cudaGetLastError();
}

template <int D, class T>
cudaError_t launch_bin(const DMesh<D, T>& M, const T* const* x, long long n, const BinBuffers& b,
                       const LaunchCfg& cfg, bool) {
    cudaError_t e = launch_bin_count<D, T>(M, x, n, b, cfg);
    if (e != cudaSuccess) return e;
    return launch_bin_rest(M.nblocks, n, b, cfg);
}

#define TB_INST_BIN(D, T)                                                                                     \
    template cudaError_t launch_bin<D, T>(const DMesh<D, T>&, const T* const*, long long, const BinBuffers&, \
                                          const LaunchCfg&, bool);                                            \
    template cudaError_t launch_bin_count<D, T>(const DMesh<D, T>&, const T* const*, long long,              \
                                                const BinBuffers&, const LaunchCfg&);
TB_INST_BIN(3, double)
TB_INST_BIN(3, float)
TB_INST_BIN(2, double)
TB_INST_BIN(2, float)

}  // namespace tb
