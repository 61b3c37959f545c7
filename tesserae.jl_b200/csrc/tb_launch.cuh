// tb_launch.cuh -- host-side launchers shared between the kernel files and the
// C-ABI layer of libtesserae_b200.so.
#pragma once

#include "tb_common.cuh"

namespace tb {

// Device buffers of one binning pass (GPUBlockStrategy arrays plus scratch).
struct BinBuffers {
    int* blockids;        // [n] caller
    int* counts;          // [nb] caller
    int* offsets;         // [nb+1] caller
    int* blocklist;       // [nb] caller
    int* perm;            // [n] caller, 1-based particle ids
    int* cursors;         // [nb] scratch
    int* perm_tmp;        // [n] scratch, 0-based ids in warp-run order
    unsigned long long* partials;  // [ntiles] scratch
    unsigned long long* sort_scratch;  // [2n] scratch for large blocks
    int* totals;          // [2] device: nactive, nassigned
};

// Scratch of a sparse grid's numbering pass (one int per block each, the scan
// partials, two totals).
struct SparseScratch {
    int* act;       // [nb] block activity
    int* offsets;   // [nb+1]
    int* cursors;   // [nb] (written by the shared scan, unused)
    unsigned long long* partials;  // [ntiles]
    int* totals;    // [2]
};

constexpr int SCAN_TILE = 1024;  // blocks per scan tile (256 threads x 4)

inline int scan_tiles(int nb) { return (nb + SCAN_TILE - 1) / SCAN_TILE; }

// Optional per-kernel timing: CUDA events recorded on the launching stream
// around every launch while profiling is enabled (tb_profile_enable).
struct Profiler {
    virtual void begin(const char* name, cudaStream_t s) = 0;
    virtual void end(cudaStream_t s) = 0;
    virtual ~Profiler() = default;
};

struct LaunchCfg {
    cudaStream_t stream;
    int num_sms;
    long long* launches;  // incremented per kernel launch
    int* err;             // device status word
    Profiler* prof;       // null unless profiling
};

// RAII scope naming the kernel launches it encloses.
struct KernelScope {
    const LaunchCfg& cfg;
    KernelScope(const LaunchCfg& c, const char* name) : cfg(c) {
        if (cfg.prof) cfg.prof->begin(name, cfg.stream);
    }
    ~KernelScope() {
        if (cfg.prof) cfg.prof->end(cfg.stream);
    }
};

template <int D, class T>
cudaError_t launch_bin(const DMesh<D, T>& M, const T* const* x, long long n, const BinBuffers& b,
                       const LaunchCfg& cfg, bool count_only_done = false);

// Count kernel alone (positions -> blockids, counts); the rest of the pass in
// launch_bin_rest. Split so a fused step can count inside G2P.
template <int D, class T>
cudaError_t launch_bin_count(const DMesh<D, T>& M, const T* const* x, long long n, const BinBuffers& b,
                             const LaunchCfg& cfg);
cudaError_t launch_bin_rest(int nblocks, long long n, const BinBuffers& b, const LaunchCfg& cfg);

// update_sparsity! from a binning pass: the node blocks within one block of a
// block that holds particles (b.blocklist / b.totals), numbered in ascending
// order into bnum (0 inactive, k >= 1), their 1-based ids into blist, the count
// into nact[0] (src/Grids/sparsity.jl:19-60, 192-232).
cudaError_t launch_sparsity(int dim, const int* nbv, int nblocks, const BinBuffers& b, const SparseScratch& sc,
                            int* bnum, int* blist, int* nact, const LaunchCfg& cfg);

// P2G scatter into a grid whose m, mv, f are already zero where it will add.
template <int D, class T, int BW>
cudaError_t launch_p2g(const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G, const Scalars<T>& s,
                       const BinBuffers& b, const LaunchCfg& cfg);

template <int D, class T>
cudaError_t launch_grid_update(const DMesh<D, T>& M, const GView<T>& G, const Scalars<T>& s, const LaunchCfg& cfg);

template <int D, class T>
cudaError_t launch_grid_zero(const DMesh<D, T>& M, const GView<T>& G, const LaunchCfg& cfg);

// With `count_next`, G2P also writes every moved particle's block id for the
// next step into b.blockids and adds it to b.counts (which the caller zeroes
// first): the count pass of the next step's binning, so that step runs
// launch_bin_rest only.
template <int D, class T, int BW>
cudaError_t launch_g2p(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                       const BinBuffers& b, const LaunchCfg& cfg, bool count_next = false);

// Sparse grid maintenance over node blocks touched now (cur) or in the previous
// transfer (prev): see tb_transfer.cu.
cudaError_t launch_mark_touched(int dim, const int* nbv, const BinBuffers& b, unsigned char* cur, int nblocks,
                                const LaunchCfg& cfg);
// The node blocks with cur or prev set, compacted into list[0 .. *count).
cudaError_t launch_touched_list(const unsigned char* cur, const unsigned char* prev, int nblocks, int* list,
                                int* count, const LaunchCfg& cfg);
template <int D, class T, int BW>
cudaError_t launch_sparse_zero(const DMesh<D, T>& M, const GView<T>& G, const int* list, const int* count,
                               const LaunchCfg& cfg);
template <int D, class T, int BW>
cudaError_t launch_sparse_grid_update(const DMesh<D, T>& M, const GView<T>& G, const Scalars<T>& s,
                                      const unsigned char* cur, const int* list, const int* count,
                                      const LaunchCfg& cfg, bool zero_after = false);

// max over the particles of sqrt((lambda + 2 mu) / (m / V)) + |v| into *out
// (the bits of a double).
template <int D, class T>
cudaError_t launch_wave_speed(const PView<T>& P, const Scalars<T>& s, unsigned long long* out, const LaunchCfg& cfg);

template <int D, class T>
cudaError_t launch_g2p_direct(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                              const LaunchCfg& cfg);

// Reverse mode: the caller's FP64 sensitivity arrays (tb_adjoint) and the
// context's FP64 grid sensitivities (component-major, nnodes each).
struct AdjView {
    double* x[3];
    double* v[3];
    double* F[9];
    double* mu;
    double* lam;
    double* B[9];  // APIC only
};
struct GradGrid {
    double* vb[3];   // d loss / d v_i (scattered by G2P backwards)
    double* vnb[3];  // d loss / d vn_i
    double* mb;      // d loss / d m_i
    double* pb[3];   // d loss / d mv_i
    double* fb[3];   // d loss / d f_i
    double* coef;    // per permutation slot: G2P backwards' scatter coefficients (2 D + D^2 arrays of n)
};

// The partition of the step being reversed (device arrays).
struct AdjPartition {
    const int* totals;     // [2] nactive, nassigned
    const int* blocklist;
    const int* offsets;
    const int* perm;
    const int* blockids;
};

// G2P, grid update and P2G backwards for one step whose forward grid is in G
// and whose partition is `part` (tb_adjoint.cu). Zeroes GB's v / vn
// sensitivities first.
template <int D, class T, int BW>
cudaError_t launch_adjoint(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                           const AdjView& A, const GradGrid& GB, const AdjPartition& part, const LaunchCfg& cfg);
// The same for WLS / KernelCorrection bases and the APIC transfer (particle-parallel,
// weight derivatives in Dual3).
template <int D, class T>
cudaError_t launch_adjoint_general(const DMesh<D, T>& M, const GView<T>& G, const PView<T>& P, const Scalars<T>& s,
                                   const AdjView& A, const GradGrid& GB, const AdjPartition& part, const LaunchCfg& cfg);

template <int D, class T>
cudaError_t launch_update_weights(const DMesh<D, T>& M, const PView<T>& P, const Scalars<T>& s, T* w, T* grad_w,
                                  long long* window, const LaunchCfg& cfg);

// reorder_particles! (tb_reorder.cu). One particle field: a device array of n
// elements of `elem` (4 or 8) bytes.
struct ReorderField {
    void* ptr;
    int elem;
};
struct ReorderArgs {
    long long n;
    int nblocks;
    int* blockids;         // [n] permuted with the particles
    int* perm;             // [n] 1-based block-sorted permutation; identity after a reorder
    const int* counts;     // [nblocks]
    const int* offsets;    // [nblocks + 1]
    double threshold;      // reorder when the score is below it (always at >= 1, never at <= 0)
    unsigned long long* acc;  // [2] scratch: same-block neighbours, non-empty blocks
    int* decision;         // [2] reorder now; reorder wanted but particles lie outside the mesh
    double* score;         // [1] contiguity score
    void* scratch;         // [n] x 8 bytes
    bool report_outside;   // raise ERR_REORDER_OUTSIDE in the status word when a reorder is refused
};
// Score and decision on the device (no host synchronisation).
cudaError_t launch_reorder_score(const ReorderArgs& a, const LaunchCfg& cfg);
// Permute `fields`, the block ids and the permutation when decision[0] is set.
cudaError_t launch_reorder_apply(const ReorderArgs& a, const ReorderField* fields, int nfields, const LaunchCfg& cfg);

}  // namespace tb
