// tb_abi.cu -- the extern "C" boundary of libtesserae_b200.so (include/tesserae_b200.h).
//
// Argument checks mirror the reference's (Tesserae.jl src/Transfer/runtime.jl:177-229,
// src/Parallel/gpu_block_strategy.jl:142-150): particle and block counts must fit
// Int32, the support window must fit the block tile, only 2D/3D meshes. Errors are
// returned as status codes with a message; no exception crosses the boundary.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>
#include <algorithm>
#include <map>

#include "tb_launch.cuh"

using namespace tb;

// Per-kernel device timing (tb_profile_enable / tb_profile_read): one pair of
// CUDA events on the launching stream around every launch of this library.
struct EventProfiler final : tb::Profiler {
    struct Span {
        const char* name;
        cudaEvent_t a, b;
    };
    std::vector<cudaEvent_t> pool;
    std::vector<Span> spans;
    const char* cur_name = nullptr;
    cudaEvent_t cur_a = nullptr;
    std::map<std::string, std::pair<long long, double>> totals;

    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    void begin(const char* name, cudaStream_t s) override {
        cur_name = name;
        cur_a = get();
        cudaEventRecord(cur_a, s);
    }
    void end(cudaStream_t s) override {
        cudaEvent_t b = get();
        cudaEventRecord(b, s);
        spans.push_back({cur_name, cur_a, b});
    }
    void collect() {
        for (auto& sp : spans) {
            cudaEventSynchronize(sp.b);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, sp.a, sp.b);
            auto& t = totals[sp.name];
            t.first += 1;
            t.second += ms;
            pool.push_back(sp.a);
            pool.push_back(sp.b);
        }
        spans.clear();
    }
    ~EventProfiler() override {
        collect();
        for (auto e : pool) cudaEventDestroy(e);
    }
};

struct tb_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    int num_sms = 148;
    long long launches = 0;
    std::string error;
    int* d_err = nullptr;            // device status word (ERR_* bits)
    int* d_totals = nullptr;         // [2] nactive, nassigned
    int* h_totals = nullptr;         // pinned mirror
    // scratch (grow-only)
    int* cursors = nullptr;
    long long cursors_cap = 0;
    int* perm_tmp = nullptr;
    long long perm_tmp_cap = 0;
    unsigned long long* partials = nullptr;
    long long partials_cap = 0;
    unsigned long long* sort_scratch = nullptr;
    long long sort_scratch_cap = 0;
    // touched node blocks of the last two transfers (sparse grid zero/update)
    // sparse grid numbering scratch
    int* sp_act = nullptr;
    long long sp_act_cap = 0;
    int* sp_off = nullptr;
    long long sp_off_cap = 0;
    int* sp_cur = nullptr;
    long long sp_cur_cap = 0;
    unsigned long long* sp_part = nullptr;
    long long sp_part_cap = 0;
    int* sp_tot = nullptr;
    long long sp_tot_cap = 0;
    unsigned char* touched_cur = nullptr;
    unsigned char* touched_prev = nullptr;
    int* touched_list = nullptr;  // [nblocks] blocks with cur or prev set, count in touched_count
    int* touched_count = nullptr;
    long long touched_cap = 0;
    const void* grid_key = nullptr;  // grid.m of the grid the flags describe
    long long grid_nblocks = 0;
    bool grid_sparse_ok = false;     // the flags describe every non-zero node of grid_key
    bool grid_dense_pending = false; // last P2G zeroed densely: the next grid half runs densely too
    bool grid_zeroed = false;        // the last grid half zeroed m, mv, f of its blocks once read
    EventProfiler* prof = nullptr;
    // context-owned state for tb_rollout_host_*
    void* roll_buf = nullptr;
    size_t roll_cap = 0;
    // reverse mode: FP64 grid sensitivities (13 components x nnodes)
    double* adj_grid = nullptr;
    long long adj_grid_cap = 0;
    double* adj_coef = nullptr;
    char* g2p2g_x = nullptr;  // tb_g2p2g_*: the new positions until the P2G half has run
    long long g2p2g_x_cap = 0;
    long long adj_coef_cap = 0;
    // checkpoint tape: states at steps 0, K, 2K, ... and one segment of K states
    char* tape_cp = nullptr;
    long long tape_cp_cap = 0;
    char* tape_seg = nullptr;
    long long tape_seg_cap = 0;
    bool tape_valid = false;
    long long tape_n = 0;
    int tape_dim = 0, tape_elem = 0;
    bool tape_apic = false, tape_x64 = false;
    int tape_nsteps = 0, tape_every = 1;
    // reorder_particles!: 8-byte-per-particle scratch, score accumulators,
    // decision words and the score
    unsigned long long* ro_scratch = nullptr;
    long long ro_scratch_cap = 0;
    unsigned long long* ro_acc = nullptr;  // [2]
    unsigned long long* wave_max = nullptr;  // tb_max_wave_speed_* result
    int* ro_decision = nullptr;            // [2]
    double* ro_score = nullptr;            // [1]
};

namespace {

int fail(tb_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->error = buf;
    return code;
}

int cuda_fail(tb_ctx* c, cudaError_t e, const char* what) {
    return fail(c, TB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

template <class P>
cudaError_t grow(P*& ptr, long long& cap, long long need) {
    if (need <= cap) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&ptr, sizeof(P) * size_t(need > 0 ? need : 1));
    if (e == cudaSuccess) cap = need;
    return e;
}

int check_ctx(tb_ctx* c) {
    if (!c) return TB_ERR_ARG;
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaSetDevice");
    return TB_OK;
}

int check_mesh(tb_ctx* c, const tb_mesh* m) {
    if (!m) return fail(c, TB_ERR_ARG, "mesh is NULL");
    if (m->dim != 2 && m->dim != 3) return fail(c, TB_ERR_UNSUPPORTED, "mesh dim %d: only 2D and 3D are supported", m->dim);
    const int bw = 1 << m->block_log2;
    if (!((m->dim == 3 && m->block_log2 == 2) || (m->dim == 2 && (m->block_log2 == 2 || m->block_log2 == 3))))
        return fail(c, TB_ERR_UNSUPPORTED, "block_size_log2 %d in %dD: supported are 2 (3D) and 2 or 3 (2D)",
                    m->block_log2, m->dim);
    long long nn = 1, nb = 1;
    for (int d = 0; d < m->dim; ++d) {
        if (m->n_nodes[d] < 2) return fail(c, TB_ERR_ARG, "mesh axis %d has %lld nodes (< 2)", d, (long long)m->n_nodes[d]);
        nn *= m->n_nodes[d];
        nb *= ((m->n_nodes[d] - 1) >> m->block_log2) + 1;
    }
    if (nb > 0x7fffffffll) return fail(c, TB_ERR_CAPACITY, "block count %lld exceeds Int32 capacity", nb);
    if (!(m->h > 0) || !(m->h_inv > 0)) return fail(c, TB_ERR_ARG, "mesh spacing must be positive");
    (void)bw;
    (void)nn;
    return TB_OK;
}

long long mesh_nblocks(const tb_mesh* m) {
    long long nb = 1;
    for (int d = 0; d < m->dim; ++d) nb *= ((m->n_nodes[d] - 1) >> m->block_log2) + 1;
    return nb;
}

// The support of every hot-path basis is 3 nodes wide; the reference checks the
// window against the block width (src/Transfer/runtime.jl:192-229).
int check_params(tb_ctx* c, const tb_step_params* p) {
    if (!p) return fail(c, TB_ERR_ARG, "params is NULL");
    if (p->basis < TB_BSPLINE_QUADRATIC || p->basis > TB_KC_UGIMP)
        return fail(c, TB_ERR_ARG, "unknown basis kind %d", p->basis);
    if (p->transfer != TB_TRANSFER_FLIP && p->transfer != TB_TRANSFER_APIC)
        return fail(c, TB_ERR_ARG, "unknown transfer kind %d", p->transfer);
    if (p->material < TB_MATERIAL_NEOHOOKEAN || p->material > TB_MATERIAL_VONMISES)
        return fail(c, TB_ERR_ARG, "unknown material %d", p->material);
    return TB_OK;
}

// x64: the FP64-position form (particles.x are double arrays, the rest T).
template <class T>
int make_pview(tb_ctx* c, const tb_particles* p, int dim, bool need_state, bool apic, PView<T>& P,
               bool x64 = false, int material = TB_MATERIAL_NEOHOOKEAN) {
    if (!p) return fail(c, TB_ERR_ARG, "particles is NULL");
    if (p->n < 0 || p->n > 0x7fffffffll)
        return fail(c, TB_ERR_CAPACITY, "particle count %lld exceeds the partition's Int32 capacity", (long long)p->n);
    std::memset(&P, 0, sizeof P);
    P.n = p->n;
    for (int d = 0; d < dim; ++d) {
        if (x64) P.x64[d] = static_cast<double*>(p->x[d]);
        else P.x[d] = static_cast<T*>(p->x[d]);
        P.v[d] = static_cast<T*>(p->v[d]);
        if (p->n && !p->x[d]) return fail(c, TB_ERR_ARG, "particles.x[%d] is NULL", d);
        if (need_state && p->n && !P.v[d]) return fail(c, TB_ERR_ARG, "particles.v[%d] is NULL", d);
    }
    P.V = static_cast<T*>(p->V);
    P.m = static_cast<const T*>(p->m);
    P.l = static_cast<const T*>(p->l);
    for (int k = 0; k < dim * dim; ++k) {
        P.gv[k] = static_cast<T*>(p->grad_v[k]);
        P.F[k] = static_cast<double*>(p->F[k]);
        P.B[k] = static_cast<T*>(p->B[k]);
        if (need_state && p->n && (!P.gv[k] || !P.F[k]))
            return fail(c, TB_ERR_ARG, "particles.grad_v/F component %d is NULL", k);
        if (apic && p->n && !P.B[k]) return fail(c, TB_ERR_ARG, "APIC transfer needs particles.B[%d]", k);
    }
    for (int k = 0; k < (dim == 3 ? 6 : 3); ++k) {
        P.sig[k] = static_cast<T*>(p->sigma[k]);
        if (need_state && p->n && !P.sig[k]) return fail(c, TB_ERR_ARG, "particles.sigma[%d] is NULL", k);
    }
    if (need_state && p->n && !P.V) return fail(c, TB_ERR_ARG, "particles.V is NULL");
    P.V0 = static_cast<const T*>(p->V0);
    P.mu = static_cast<const T*>(p->mu);
    P.lam = static_cast<const T*>(p->lambda);
    P.eps_p = static_cast<T*>(p->eps_p);
    for (int k = 0; k < 6; ++k) P.Cp_inv[k] = static_cast<T*>(p->Cp_inv[k]);
    if (need_state && material == TB_MATERIAL_VONMISES) {
        if (dim != 3) return fail(c, TB_ERR_UNSUPPORTED, "the von Mises model is three-dimensional");
        if (p->n && !P.eps_p) return fail(c, TB_ERR_ARG, "the von Mises model needs particles.eps_p");
        for (int k = 0; k < 6; ++k)
            if (p->n && !P.Cp_inv[k]) return fail(c, TB_ERR_ARG, "the von Mises model needs particles.Cp_inv[%d]", k);
    }
    return TB_OK;
}

template <class T>
int make_gview(tb_ctx* c, const tb_grid* g, int dim, GView<T>& G, int block_log2 = 0) {
    if (!g) return fail(c, TB_ERR_ARG, "grid is NULL");
    std::memset(&G, 0, sizeof G);
    G.m = static_cast<T*>(g->m);
    if (!G.m) return fail(c, TB_ERR_ARG, "grid.m is NULL");
    for (int d = 0; d < dim; ++d) {
        G.mv[d] = static_cast<T*>(g->mv[d]);
        G.f[d] = static_cast<T*>(g->f[d]);
        G.v[d] = static_cast<T*>(g->v[d]);
        G.vn[d] = static_cast<T*>(g->vn[d]);
        if (!G.mv[d] || !G.f[d] || !G.v[d] || !G.vn[d]) return fail(c, TB_ERR_ARG, "grid component %d is NULL", d);
    }
    if (g->block_numbering || g->active_blocks || g->nactive) {  // block-sparse grid
        if (!g->block_numbering || !g->active_blocks || !g->nactive)
            return fail(c, TB_ERR_ARG, "a sparse grid needs block_numbering, active_blocks and nactive");
        const long long bl = 1ll << (block_log2 * dim);
        if (g->capacity < 0 || g->capacity % bl != 0)
            return fail(c, TB_ERR_ARG, "sparse grid capacity %lld is not a multiple of the block length %lld",
                        (long long)g->capacity, bl);
        G.bnum = g->block_numbering;
        G.blist = g->active_blocks;
        G.nact = g->nactive;
        G.cap = g->capacity;
        G.L = block_log2;
    }
    return TB_OK;
}

int sparse_scratch(tb_ctx* c, long long nb, SparseScratch& sc) {
    cudaError_t e;
    if ((e = grow(c->sp_act, c->sp_act_cap, nb)) != cudaSuccess ||
        (e = grow(c->sp_off, c->sp_off_cap, nb + 1)) != cudaSuccess ||
        (e = grow(c->sp_cur, c->sp_cur_cap, nb)) != cudaSuccess ||
        (e = grow(c->sp_part, c->sp_part_cap, scan_tiles(int(nb)))) != cudaSuccess ||
        (e = grow(c->sp_tot, c->sp_tot_cap, 2)) != cudaSuccess)
        return cuda_fail(c, e, "cudaMalloc sparse grid scratch");
    sc = SparseScratch{c->sp_act, c->sp_off, c->sp_cur, c->sp_part, c->sp_tot};
    return TB_OK;
}

int bin_buffers(tb_ctx* c, const tb_partition* part, long long n, long long nb, BinBuffers& B) {
    if (!part) return fail(c, TB_ERR_ARG, "partition is NULL");
    if (part->nblocks != nb)
        return fail(c, TB_ERR_ARG, "partition.nblocks %lld does not match the mesh (%lld)", (long long)part->nblocks, nb);
    if (!part->counts || !part->offsets || !part->blocklist || (n && (!part->blockids || !part->particleindices)))
        return fail(c, TB_ERR_ARG, "partition array is NULL");
    cudaError_t e;
    if ((e = grow(c->cursors, c->cursors_cap, nb)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc cursors");
    if ((e = grow(c->perm_tmp, c->perm_tmp_cap, n)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc perm_tmp");
    if ((e = grow(c->partials, c->partials_cap, scan_tiles(int(nb)))) != cudaSuccess)
        return cuda_fail(c, e, "cudaMalloc partials");
    if ((e = grow(c->sort_scratch, c->sort_scratch_cap, 2 * n)) != cudaSuccess)
        return cuda_fail(c, e, "cudaMalloc sort scratch");
    B.blockids = part->blockids;
    B.counts = part->counts;
    B.offsets = part->offsets;
    B.blocklist = part->blocklist;
    B.perm = part->particleindices;
    B.cursors = c->cursors;
    B.perm_tmp = c->perm_tmp;
    B.partials = c->partials;
    B.sort_scratch = c->sort_scratch;
    B.totals = c->d_totals;
    return TB_OK;
}

LaunchCfg cfg_of(tb_ctx* c) { return LaunchCfg{c->stream, c->num_sms, &c->launches, c->d_err, c->prof}; }

// Reads and clears the device status word (synchronises the stream).
int check_device_status(tb_ctx* c) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "device status readback");
    if (h) {
        cudaMemsetAsync(c->d_err, 0, sizeof(int), c->stream);
        std::string why;
        if (h & ERR_TILE_RANGE) why += " support window outside its block tile;";
        if (h & ERR_GIMP_LENGTH) why += " uGIMP requires 0 <= l <= spacing(mesh);";
        if (h & ERR_WLS_SINGULAR) why += " singular WLS moment matrix;";
        if (h & ERR_REORDER_OUTSIDE)
            why += " reorder_particles!: some particles are outside the mesh and were not assigned to any block;";
        if (h & ERR_INACTIVE_NODE)
            why += " @P2G: a support node of an inactive sparse-grid block (run update_sparsity for these positions);";
        if (h & ERR_SPGRID_CAPACITY) why += " the sparse grid's active blocks exceed its field arrays' capacity;";
        return fail(c, TB_ERR_DEVICE, "kernel reported:%s", why.c_str());
    }
    return TB_OK;
}

// Every particle field present in `p` with its element size (x is double in
// the FP64-position form, F always double, the rest the state scalar).
int particle_fields(const tb_particles* p, int D, size_t elem, bool x64, std::vector<ReorderField>& out) {
    out.clear();
    auto add = [&](void* ptr, size_t e) {
        if (ptr) out.push_back({ptr, int(e)});
    };
    for (int d = 0; d < D; ++d) add(p->x[d], x64 ? sizeof(double) : elem);
    for (int d = 0; d < D; ++d) add(p->v[d], elem);
    add(p->V, elem);
    add(p->m, elem);
    add(p->l, elem);
    for (int k = 0; k < D * D; ++k) add(p->grad_v[k], elem);
    for (int k = 0; k < (D == 3 ? 6 : 3); ++k) add(p->sigma[k], elem);
    for (int k = 0; k < D * D; ++k) add(p->F[k], sizeof(double));
    for (int k = 0; k < D * D; ++k) add(p->B[k], elem);
    add(p->V0, elem);
    add(p->mu, elem);
    add(p->lambda, elem);
    add(p->eps_p, elem);
    for (int k = 0; k < (D == 3 ? 6 : 3); ++k) add(p->Cp_inv[k], elem);
    return TB_OK;
}

int reorder_args(tb_ctx* c, const tb_partition* part, long long n, double threshold, ReorderArgs& a) {
    if (!part || (n && (!part->blockids || !part->particleindices)) || !part->counts || !part->offsets)
        return fail(c, TB_ERR_ARG, "partition array is NULL");
    cudaError_t e;
    if ((e = grow(c->ro_scratch, c->ro_scratch_cap, n)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc reorder");
    if (!c->ro_acc) {
        if ((e = cudaMalloc(&c->ro_acc, 2 * sizeof(unsigned long long))) != cudaSuccess ||
            (e = cudaMalloc(&c->ro_decision, 2 * sizeof(int))) != cudaSuccess ||
            (e = cudaMalloc(&c->ro_score, sizeof(double))) != cudaSuccess)
            return cuda_fail(c, e, "cudaMalloc reorder words");
    }
    a = ReorderArgs{};
    a.n = n;
    a.nblocks = int(part->nblocks);
    a.blockids = part->blockids;
    a.perm = part->particleindices;
    a.counts = part->counts;
    a.offsets = part->offsets;
    a.threshold = threshold;
    a.acc = c->ro_acc;
    a.decision = c->ro_decision;
    a.score = c->ro_score;
    a.scratch = c->ro_scratch;
    a.report_outside = true;
    return TB_OK;
}

int touched_buffers(tb_ctx* c, long long nb) {
    cudaError_t e;
    if (nb > c->touched_cap) {
        long long cap = c->touched_cap;
        if ((e = grow(c->touched_cur, cap, nb)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc touched flags");
        cap = c->touched_cap;
        if ((e = grow(c->touched_prev, cap, nb)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc touched flags");
        cap = c->touched_cap;
        if ((e = grow(c->touched_list, cap, nb)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc touched list");
        long long one = c->touched_count ? 1 : 0;
        if ((e = grow(c->touched_count, one, 1)) != cudaSuccess) return cuda_fail(c, e, "cudaMalloc touched count");
        c->touched_cap = nb;
        c->grid_sparse_ok = false;
    }
    return TB_OK;
}

// Zero the P2G targets where this transfer adds, then scatter. The first
// transfer of an ABI call zeroes every node of the grid (its content is the
// caller's); the following steps of the same call zero only the node blocks
// touched by this or the previous step, which are the only ones that can be
// non-zero, so the grid matches the reference's dense fillzero!
// (src/Core/zero.jl:100-106) at a fraction of the traffic. Nothing is cached
// across calls: a later grid may reuse an earlier grid's address.
template <int D, class T, int BW>
cudaError_t p2g_with_zero(tb_ctx* c, const DMesh<D, T>& M, const PView<T>& P, const GView<T>& G,
                          const Scalars<T>& S, const BinBuffers& B, const LaunchCfg& cfg) {
    if (G.bnum) {  // block-sparse grid: zero the stored nodes, scatter
        c->grid_sparse_ok = false;
        c->grid_zeroed = false;
        cudaError_t e = launch_grid_zero<D, T>(M, G, cfg);
        return e == cudaSuccess ? launch_p2g<D, T, BW>(M, P, G, S, B, cfg) : e;
    }
    const bool known = c->grid_sparse_ok && c->grid_key == G.m && c->grid_nblocks == M.nblocks;
    // after a grid half that zeroed its blocks once read, every P2G target is zero
    const bool zeroed = known && c->grid_zeroed;
    c->grid_zeroed = false;
    std::swap(c->touched_cur, c->touched_prev);
    cudaError_t e = cudaMemsetAsync(c->touched_cur, 0, size_t(M.nblocks), cfg.stream);
    if (e == cudaSuccess && !known) e = cudaMemsetAsync(c->touched_prev, 0, size_t(M.nblocks), cfg.stream);
    if (e == cudaSuccess) e = launch_mark_touched(D, M.nb, B, c->touched_cur, M.nblocks, cfg);
    if (e == cudaSuccess)
        e = launch_touched_list(c->touched_cur, c->touched_prev, M.nblocks, c->touched_list, c->touched_count, cfg);
    if (e == cudaSuccess && !zeroed)
        e = known ? launch_sparse_zero<D, T, BW>(M, G, c->touched_list, c->touched_count, cfg)
                  : launch_grid_zero<D, T>(M, G, cfg);
    if (e == cudaSuccess) e = launch_p2g<D, T, BW>(M, P, G, S, B, cfg);
    c->grid_key = G.m;
    c->grid_nblocks = M.nblocks;
    c->grid_sparse_ok = (e == cudaSuccess);
    c->grid_dense_pending = !known;
    return e;
}

// Grid half: over the touched node blocks when the flags describe this grid
// (zeroing v and vn of blocks touched only before), else over every node. With
// zero_after (a later step of the same call scatters into this grid again, so
// the caller cannot see m, mv, f in between) the sparse half also zeroes m, mv,
// f of the blocks it reads, and the next P2G skips its zero pass.
template <int D, class T, int BW>
cudaError_t grid_update_sparse_or_dense(tb_ctx* c, const DMesh<D, T>& M, const GView<T>& G, const Scalars<T>& S,
                                        const LaunchCfg& cfg, bool zero_after = false) {
    if (G.bnum) return launch_grid_update<D, T>(M, G, S, cfg);  // over the stored nodes
    const bool known = c->grid_sparse_ok && c->grid_key == G.m && c->grid_nblocks == M.nblocks &&
                       !c->grid_dense_pending;
    c->grid_dense_pending = false;
    c->grid_zeroed = false;
    if (known) {
        const cudaError_t e = launch_sparse_grid_update<D, T, BW>(M, G, S, c->touched_cur, c->touched_list,
                                                                  c->touched_count, cfg, zero_after);
        c->grid_zeroed = zero_after && e == cudaSuccess;
        return e;
    }
    return launch_grid_update<D, T>(M, G, S, cfg);
}

template <int D, class T, int BW>
int run_step(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
             const tb_step_params* prm, int nsteps, bool do_bin, bool do_p2g, bool do_grid, bool do_g2p,
             bool x64 = false, double reorder_threshold = 0.0) {
    auto M = make_dmesh<D, T>(*m);
    auto S = make_scalars<T>(*prm);
    PView<T> P;
    GView<T> G;
    int rc;
    if ((rc = make_pview<T>(c, p, D, true, prm->transfer == TB_TRANSFER_APIC, P, x64, prm->material)) != TB_OK)
        return rc;
    if ((rc = make_gview<T>(c, g, D, G, m->block_log2)) != TB_OK) return rc;
    BinBuffers B;
    if ((rc = bin_buffers(c, part, P.n, M.nblocks, B)) != TB_OK) return rc;
    const LaunchCfg cfg = cfg_of(c);
    const T* xs[3] = {P.x[0], P.x[1], D == 3 ? P.x[2] : P.x[1]};
    // FP64 positions are binned by the FP64 findblock (the reference's Float64 rule)
    const auto M64 = make_dmesh<D, double>(*m);
    const double* xs64[3] = {P.x64[0], P.x64[1], D == 3 ? P.x64[2] : P.x64[1]};
    cudaError_t e = cudaSuccess;
    if ((do_p2g || do_grid) && (rc = touched_buffers(c, M.nblocks)) != TB_OK) return rc;
    // reorder_particles!(particles, partition; threshold) after every binning
    // (the loop of docs/literate/tutorials/taylor_impact.jl:120-127)
    const bool reorder = do_bin && reorder_threshold > 0.0;
    std::vector<ReorderField> fields;
    ReorderArgs RA{};
    if (reorder) {
        particle_fields(p, D, sizeof(T), x64, fields);
        if ((rc = reorder_args(c, part, P.n, reorder_threshold, RA)) != TB_OK) return rc;
    }
    c->grid_sparse_ok = false;  // the first step of every call runs densely
    c->grid_zeroed = false;
    // Inside one call, the G2P of step s counts the particles into blocks for
    // step s + 1 (the count pass of its binning); the last step does not, so the
    // partition left to the caller is the last step's own.
    bool counted = false;
    SparseScratch SC{};
    if (G.bnum && do_bin && (rc = sparse_scratch(c, M.nblocks, SC)) != TB_OK) return rc;
    for (int s = 0; s < nsteps && e == cudaSuccess; ++s) {
        if (do_bin) {
            if (counted) e = launch_bin_rest(M.nblocks, P.n, B, cfg);
            else e = x64 ? launch_bin<D, double>(M64, xs64, P.n, B, cfg) : launch_bin<D, T>(M, xs, P.n, B, cfg);
            // a sparse grid follows the particles: update_sparsity! every step
            if (e == cudaSuccess && G.bnum)
                e = launch_sparsity(D, M.nb, M.nblocks, B, SC, g->block_numbering, g->active_blocks, g->nactive, cfg);
        }
        const bool count_next = do_bin && do_g2p && s + 1 < nsteps;
        counted = false;
        if (e == cudaSuccess && reorder) e = launch_reorder_score(RA, cfg);
        if (e == cudaSuccess && reorder) e = launch_reorder_apply(RA, fields.data(), int(fields.size()), cfg);
        if (e == cudaSuccess && do_p2g) e = p2g_with_zero<D, T, BW>(c, M, P, G, S, B, cfg);
        if (e == cudaSuccess && do_grid)
            e = grid_update_sparse_or_dense<D, T, BW>(c, M, G, S, cfg, do_p2g && s + 1 < nsteps);
        if (e == cudaSuccess && do_g2p) {
            e = launch_g2p<D, T, BW>(M, G, P, S, B, cfg, count_next);
            counted = count_next;
        }
    }
    c->grid_zeroed = false;  // a P2G outside this call zeroes for itself
    if (e != cudaSuccess) return cuda_fail(c, e, "kernel launch");
    return TB_OK;
}

template <class T>
int dispatch_step(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                  const tb_step_params* prm, int nsteps, bool b, bool p2g, bool gr, bool g2p, bool x64 = false,
                  double reorder_threshold = 0.0) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_mesh(c, m)) != TB_OK) return rc;
    if ((rc = check_params(c, prm)) != TB_OK) return rc;
    if (nsteps < 0) return fail(c, TB_ERR_ARG, "nsteps must be >= 0");
    if (x64 && m->dim != 3 && (prm->transfer != TB_TRANSFER_FLIP || prm->basis == TB_WLS_BSPLINE_QUADRATIC ||
                               prm->basis == TB_WLS_UGIMP))
        return fail(c, TB_ERR_UNSUPPORTED, "the FP64-position form runs WLS and APIC in 3D only");
    if (!(reorder_threshold >= 0.0 && reorder_threshold <= 1.0))
        return fail(c, TB_ERR_ARG, "reorder threshold must be in [0, 1]");
    if (m->dim == 3) return run_step<3, T, 4>(c, m, p, part, g, prm, nsteps, b, p2g, gr, g2p, x64, reorder_threshold);
    if (m->block_log2 == 3)
        return run_step<2, T, 8>(c, m, p, part, g, prm, nsteps, b, p2g, gr, g2p, x64, reorder_threshold);
    return run_step<2, T, 4>(c, m, p, part, g, prm, nsteps, b, p2g, gr, g2p, x64, reorder_threshold);
}

// reorder_particles!(particles, partition; threshold) on its own: the partition
// must come from binning these particles. Synchronous (returns whether it
// reordered); particles outside the mesh are an error when a reorder is due, as
// on the reference's GPU path (gpu_block_strategy.jl:213-216).
int do_reorder(tb_ctx* c, tb_particles* p, tb_partition* part, int dim, size_t elem, bool x64, double threshold,
               int32_t* reordered, double* score) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if (!p) return fail(c, TB_ERR_ARG, "particles is NULL");
    if (dim != 2 && dim != 3) return fail(c, TB_ERR_ARG, "dim must be 2 or 3");
    if (!(threshold >= 0.0 && threshold <= 1.0)) return fail(c, TB_ERR_ARG, "threshold must be in [0, 1]");
    if (p->n < 0 || p->n > 0x7fffffffll) return fail(c, TB_ERR_CAPACITY, "particle count exceeds Int32 capacity");
    for (int d = 0; d < dim; ++d)
        if (p->n && !p->x[d]) return fail(c, TB_ERR_ARG, "particles.x[%d] is NULL", d);
    std::vector<ReorderField> fields;
    particle_fields(p, dim, elem, x64, fields);
    ReorderArgs RA{};
    if ((rc = reorder_args(c, part, p->n, threshold, RA)) != TB_OK) return rc;
    RA.report_outside = false;
    const LaunchCfg cfg = cfg_of(c);
    cudaError_t e = launch_reorder_score(RA, cfg);
    if (e == cudaSuccess) e = launch_reorder_apply(RA, fields.data(), int(fields.size()), cfg);
    int dec[2] = {0, 0};
    double sc = 1.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(dec, c->ro_decision, sizeof dec, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sc, c->ro_score, sizeof sc, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "reorder");
    if (reordered) *reordered = dec[0];
    if (score) *score = sc;
    if (dec[1])
        return fail(c, TB_ERR_ARG, "reorder_particles!: some particles are outside the mesh and were not assigned "
                                   "to any block; filter them out before reordering on GPU");
    return TB_OK;
}

template <class T>
int do_bin_only(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part, int64_t* nactive,
                int64_t* nassigned) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_mesh(c, m)) != TB_OK) return rc;
    PView<T> P;
    if ((rc = make_pview<T>(c, p, m->dim, false, false, P)) != TB_OK) return rc;
    BinBuffers B;
    if ((rc = bin_buffers(c, part, P.n, mesh_nblocks(m), B)) != TB_OK) return rc;
    const LaunchCfg cfg = cfg_of(c);
    const T* xs[3] = {P.x[0], P.x[1], m->dim == 3 ? P.x[2] : P.x[1]};
    cudaError_t e = (m->dim == 3) ? launch_bin<3, T>(make_dmesh<3, T>(*m), xs, P.n, B, cfg)
                                  : launch_bin<2, T>(make_dmesh<2, T>(*m), xs, P.n, B, cfg);
    if (e != cudaSuccess) return cuda_fail(c, e, "binning launch");
    e = cudaMemcpyAsync(c->h_totals, c->d_totals, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "binning totals readback");
    if (nactive) *nactive = c->h_totals[0];
    if (nassigned) *nassigned = c->h_totals[1];
    return TB_OK;
}

// update_sparsity!(grid, particles.x): bin, number the active node blocks, read
// the count back (src/Grids/sparsity.jl:19-60; the reference also reads its
// active count back to size SpArray.data) and zero the stored fields.
template <int D, class T>
int sparsity_impl(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part, tb_grid* g,
                  int64_t* nstored, bool x64) {
    PView<T> P;
    int rc;
    if ((rc = make_pview<T>(c, p, D, false, false, P, x64)) != TB_OK) return rc;
    if (!g || !g->block_numbering || !g->active_blocks || !g->nactive)
        return fail(c, TB_ERR_ARG, "update_sparsity needs a sparse grid (block_numbering, active_blocks, nactive)");
    const auto M = make_dmesh<D, T>(*m);
    BinBuffers B;
    if ((rc = bin_buffers(c, part, P.n, M.nblocks, B)) != TB_OK) return rc;
    SparseScratch SC;
    if ((rc = sparse_scratch(c, M.nblocks, SC)) != TB_OK) return rc;
    const LaunchCfg cfg = cfg_of(c);
    const T* xs[3] = {P.x[0], P.x[1], D == 3 ? P.x[2] : P.x[1]};
    const double* xs64[3] = {P.x64[0], P.x64[1], D == 3 ? P.x64[2] : P.x64[1]};
    cudaError_t e = x64 ? launch_bin<D, double>(make_dmesh<D, double>(*m), xs64, P.n, B, cfg)
                        : launch_bin<D, T>(M, xs, P.n, B, cfg);
    if (e == cudaSuccess)
        e = launch_sparsity(D, M.nb, M.nblocks, B, SC, g->block_numbering, g->active_blocks, g->nactive, cfg);
    if (e != cudaSuccess) return cuda_fail(c, e, "update_sparsity launch");
    e = cudaMemcpyAsync(c->h_totals, g->nactive, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "sparse grid count readback");
    const long long need = (long long)c->h_totals[0] << (m->block_log2 * D);
    if (nstored) *nstored = need;
    if (need > g->capacity)
        return fail(c, TB_ERR_CAPACITY, "the sparse grid needs %lld nodes per field, its arrays hold %lld", need,
                    (long long)g->capacity);
    // the renumbered storage starts zero (SpArray data after update_sparsity!)
    void* fields[1 + 4 * 3] = {g->m};
    for (int d = 0; d < D; ++d) {
        fields[1 + d] = g->mv[d];
        fields[1 + D + d] = g->f[d];
        fields[1 + 2 * D + d] = g->v[d];
        fields[1 + 3 * D + d] = g->vn[d];
    }
    for (int i = 0; i < 1 + 4 * D && e == cudaSuccess; ++i)
        e = fields[i] ? cudaMemsetAsync(fields[i], 0, sizeof(T) * size_t(need), c->stream) : cudaErrorInvalidValue;
    if (e != cudaSuccess) return cuda_fail(c, e, "sparse grid zero fill");
    return TB_OK;
}

template <class T>
int do_update_sparsity(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part, tb_grid* g,
                       int64_t* nstored, bool x64 = false) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_mesh(c, m)) != TB_OK) return rc;
    if (m->dim == 3) return sparsity_impl<3, T>(c, m, p, part, g, nstored, x64);
    return sparsity_impl<2, T>(c, m, p, part, g, nstored, x64);
}

template <class T>
int do_weights(tb_ctx* c, const tb_mesh* m, const tb_particles* p, const tb_step_params* prm, tb_weights* w) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_mesh(c, m)) != TB_OK) return rc;
    if ((rc = check_params(c, prm)) != TB_OK) return rc;
    if (!w || (p && p->n && (!w->w || !w->grad_w || !w->window))) return fail(c, TB_ERR_ARG, "weights array is NULL");
    PView<T> P;
    if ((rc = make_pview<T>(c, p, m->dim, false, false, P)) != TB_OK) return rc;
    auto S = make_scalars<T>(*prm);
    const LaunchCfg cfg = cfg_of(c);
    cudaError_t e;
    if (m->dim == 3)
        e = launch_update_weights<3, T>(make_dmesh<3, T>(*m), P, S, static_cast<T*>(w->w), static_cast<T*>(w->grad_w),
                                        reinterpret_cast<long long*>(w->window), cfg);
    else
        e = launch_update_weights<2, T>(make_dmesh<2, T>(*m), P, S, static_cast<T*>(w->w), static_cast<T*>(w->grad_w),
                                        reinterpret_cast<long long*>(w->window), cfg);
    if (e != cudaSuccess) return cuda_fail(c, e, "update_weights launch");
    return TB_OK;
}

template <class T>
int do_grid_update(tb_ctx* c, const tb_mesh* m, tb_grid* g, const tb_step_params* prm) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK || (rc = check_mesh(c, m)) != TB_OK || (rc = check_params(c, prm)) != TB_OK)
        return rc;
    const LaunchCfg cfg = cfg_of(c);
    cudaError_t e;
    GView<T> G;
    if ((rc = make_gview<T>(c, g, m->dim, G, m->block_log2)) != TB_OK) return rc;
    c->grid_sparse_ok = false;  // a standalone call cannot know which nodes are non-zero
    if (m->dim == 3)
        e = grid_update_sparse_or_dense<3, T, 4>(c, make_dmesh<3, T>(*m), G, make_scalars<T>(*prm), cfg);
    else if (m->block_log2 == 3)
        e = grid_update_sparse_or_dense<2, T, 8>(c, make_dmesh<2, T>(*m), G, make_scalars<T>(*prm), cfg);
    else
        e = grid_update_sparse_or_dense<2, T, 4>(c, make_dmesh<2, T>(*m), G, make_scalars<T>(*prm), cfg);
    return e == cudaSuccess ? TB_OK : cuda_fail(c, e, "grid update launch");
}

template <class T>
int do_g2p_direct(tb_ctx* c, const tb_mesh* m, const tb_grid* g, tb_particles* p, const tb_step_params* prm) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK || (rc = check_mesh(c, m)) != TB_OK || (rc = check_params(c, prm)) != TB_OK)
        return rc;
    PView<T> P;
    GView<T> G;
    if ((rc = make_pview<T>(c, p, m->dim, true, prm->transfer == TB_TRANSFER_APIC, P, false, prm->material)) !=
        TB_OK)
        return rc;
    if ((rc = make_gview<T>(c, g, m->dim, G, m->block_log2)) != TB_OK) return rc;
    const LaunchCfg cfg = cfg_of(c);
    cudaError_t e = (m->dim == 3) ? launch_g2p_direct<3, T>(make_dmesh<3, T>(*m), G, P, make_scalars<T>(*prm), cfg)
                                  : launch_g2p_direct<2, T>(make_dmesh<2, T>(*m), G, P, make_scalars<T>(*prm), cfg);
    return e == cudaSuccess ? TB_OK : cuda_fail(c, e, "g2p launch");
}

// Host-buffer rollout: stage the particle state into a context-owned device
// block, run the steps on a context-owned grid and partition, copy back.
template <class T>
int do_rollout(tb_ctx* c, const tb_mesh* m, tb_particles* host, const tb_step_params* prm, int nsteps,
               bool x64 = false) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_mesh(c, m)) != TB_OK) return rc;
    if ((rc = check_params(c, prm)) != TB_OK) return rc;
    if (!host) return fail(c, TB_ERR_ARG, "particles is NULL");
    const int D = m->dim;
    const long long n = host->n;
    if (n < 0 || n > 0x7fffffffll) return fail(c, TB_ERR_CAPACITY, "particle count exceeds Int32 capacity");
    const bool apic = prm->transfer == TB_TRANSFER_APIC;
    long long nn = 1;
    for (int d = 0; d < D; ++d) nn *= m->n_nodes[d];
    const long long nb = mesh_nblocks(m);
    // Fields moved: x, v, V, grad_v, sigma (T); F (double); optional m, l, B, V0, mu, lambda (T), and the
    // von Mises state eps_p, Cp_inv (T, in and out).
    // in: copied to the device before the steps; out: copied back after them.
    // grad_v is written for every particle by every G2P and read by no step, so
    // it is copied out only.
    struct Field {
        void** host_slot;
        size_t elem;
        bool inout;
        bool in = true;
    };
    std::vector<Field> fields;
    auto add = [&](void** slot, size_t elem, bool inout, bool in = true) {
        if (*slot) fields.push_back({slot, elem, inout, in});
    };
    for (int d = 0; d < D; ++d) add(&host->x[d], x64 ? sizeof(double) : sizeof(T), true);
    for (int d = 0; d < D; ++d) add(&host->v[d], sizeof(T), true);
    add(&host->V, sizeof(T), true);
    for (int k = 0; k < D * D; ++k) add(&host->grad_v[k], sizeof(T), true, nsteps == 0);
    for (int k = 0; k < (D == 3 ? 6 : 3); ++k) add(&host->sigma[k], sizeof(T), true);
    for (int k = 0; k < D * D; ++k) add(&host->F[k], sizeof(double), true);
    if (apic)
        for (int k = 0; k < D * D; ++k) add(&host->B[k], sizeof(T), true);
    add(&host->m, sizeof(T), false);
    add(&host->l, sizeof(T), false);
    add(&host->V0, sizeof(T), false);
    add(&host->mu, sizeof(T), false);
    add(&host->lambda, sizeof(T), false);
    if (prm->material == TB_MATERIAL_VONMISES) {
        add(&host->eps_p, sizeof(T), true);
        for (int k = 0; k < (D == 3 ? 6 : 3); ++k) add(&host->Cp_inv[k], sizeof(T), true);
    }
    auto align = [](size_t v) { return (v + 255) & ~size_t(255); };
    size_t bytes = 0;
    for (auto& f : fields) bytes += align(f.elem * size_t(n));
    const size_t grid_bytes = align(sizeof(T) * size_t(nn)) * size_t(1 + 4 * D);
    const size_t part_bytes = align(sizeof(int) * size_t(n)) * 2 + align(sizeof(int) * size_t(nb)) * 2 +
                              align(sizeof(int) * size_t(nb + 1));
    const size_t total = bytes + grid_bytes + part_bytes;
    if (total > c->roll_cap) {
        if (c->roll_buf) cudaFree(c->roll_buf);
        c->roll_buf = nullptr;
        c->roll_cap = 0;
        cudaError_t e = cudaMalloc(&c->roll_buf, total);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc rollout state");
        c->roll_cap = total;
        e = cudaMemsetAsync(c->roll_buf, 0, total, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaMemsetAsync rollout state");
    }
    char* base = static_cast<char*>(c->roll_buf);
    tb_particles dev = *host;
    size_t off = 0;
    std::vector<void*> dptr(fields.size());
    for (size_t i = 0; i < fields.size(); ++i) {
        dptr[i] = base + off;
        off += align(fields[i].elem * size_t(n));
    }
    // device particle struct mirrors host with device pointers
    {
        size_t i = 0;
        auto remap = [&](void** hs) {
            for (size_t k = 0; k < fields.size(); ++k)
                if (fields[k].host_slot == hs) return dptr[k];
            return (void*)nullptr;
        };
        for (int d = 0; d < D; ++d) dev.x[d] = remap(&host->x[d]);
        for (int d = 0; d < D; ++d) dev.v[d] = remap(&host->v[d]);
        dev.V = remap(&host->V);
        for (int k = 0; k < D * D; ++k) dev.grad_v[k] = remap(&host->grad_v[k]);
        for (int k = 0; k < (D == 3 ? 6 : 3); ++k) dev.sigma[k] = remap(&host->sigma[k]);
        for (int k = 0; k < D * D; ++k) dev.F[k] = remap(&host->F[k]);
        for (int k = 0; k < D * D; ++k) dev.B[k] = apic ? remap(&host->B[k]) : nullptr;
        dev.m = remap(&host->m);
        dev.l = remap(&host->l);
        dev.V0 = remap(&host->V0);
        dev.mu = remap(&host->mu);
        dev.lambda = remap(&host->lambda);
        dev.eps_p = remap(&host->eps_p);
        for (int k = 0; k < 6; ++k) dev.Cp_inv[k] = k < (D == 3 ? 6 : 3) ? remap(&host->Cp_inv[k]) : nullptr;
        (void)i;
    }
    tb_grid g{};
    g.m = base + off;
    off += align(sizeof(T) * size_t(nn));
    for (int d = 0; d < D; ++d) {
        g.mv[d] = base + off;
        off += align(sizeof(T) * size_t(nn));
        g.f[d] = base + off;
        off += align(sizeof(T) * size_t(nn));
        g.v[d] = base + off;
        off += align(sizeof(T) * size_t(nn));
        g.vn[d] = base + off;
        off += align(sizeof(T) * size_t(nn));
    }
    tb_partition part{};
    part.blockids = reinterpret_cast<int32_t*>(base + off);
    off += align(sizeof(int) * size_t(n));
    part.particleindices = reinterpret_cast<int32_t*>(base + off);
    off += align(sizeof(int) * size_t(n));
    part.counts = reinterpret_cast<int32_t*>(base + off);
    off += align(sizeof(int) * size_t(nb));
    part.blocklist = reinterpret_cast<int32_t*>(base + off);
    off += align(sizeof(int) * size_t(nb));
    part.offsets = reinterpret_cast<int32_t*>(base + off);
    part.nblocks = nb;
    cudaError_t e = cudaSuccess;
    for (size_t i = 0; i < fields.size() && e == cudaSuccess; ++i)
        if (fields[i].in)
            e = cudaMemcpyAsync(dptr[i], *fields[i].host_slot, fields[i].elem * size_t(n), cudaMemcpyHostToDevice,
                                c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "rollout H2D");
    rc = dispatch_step<T>(c, m, &dev, &part, &g, prm, nsteps, true, true, true, true, x64);
    if (rc != TB_OK) return rc;
    for (size_t i = 0; i < fields.size() && e == cudaSuccess; ++i)
        if (fields[i].inout)
            e = cudaMemcpyAsync(*fields[i].host_slot, dptr[i], fields[i].elem * size_t(n), cudaMemcpyDeviceToHost,
                                c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "rollout D2H");
    return check_device_status(c);
}

template <class T>
int do_wave_speed(tb_ctx* c, int32_t dim, const tb_particles* p, const tb_step_params* prm, double* cmax) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_params(c, prm)) != TB_OK) return rc;
    if (dim != 2 && dim != 3) return fail(c, TB_ERR_ARG, "dim must be 2 or 3");
    if (!cmax) return fail(c, TB_ERR_ARG, "c_max is NULL");
    PView<T> P;
    if ((rc = make_pview<T>(c, p, dim, false, false, P)) != TB_OK) return rc;
    if (P.n && !P.V) return fail(c, TB_ERR_ARG, "particles.V is NULL");
    for (int d = 0; d < dim; ++d)
        if (P.n && !P.v[d]) return fail(c, TB_ERR_ARG, "particles.v[%d] is NULL", d);
    cudaError_t e = cudaSuccess;
    if (!c->wave_max) e = cudaMalloc(&c->wave_max, sizeof(unsigned long long));
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc wave speed");
    const auto S = make_scalars<T>(*prm);
    e = dim == 3 ? launch_wave_speed<3, T>(P, S, c->wave_max, cfg_of(c)) : launch_wave_speed<2, T>(P, S, c->wave_max, cfg_of(c));
    unsigned long long bits = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, c->wave_max, sizeof bits, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "wave speed");
    std::memcpy(cmax, &bits, sizeof bits);
    return TB_OK;
}

// @G2P2G for the FLIP/PIC equation set (src/Transfer/g2p2g.jl:98-159): the
// particles are binned at their current positions; G2P runs with its new
// positions going to context scratch, so the P2G half (m, mv, f, zeroed first)
// still weighs every particle at the position it had before the G2P half
// moved it, as the reference binds one support window for both halves
// (g2p2g.jl:103-106), and reads the updated v, sigma, V; the grid half follows;
// the new positions then replace x.
template <int D, class T, int BW>
int g2p2g_impl(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
               const tb_step_params* prm, bool x64) {
    const auto M = make_dmesh<D, T>(*m);
    const auto S = make_scalars<T>(*prm);
    PView<T> P;
    GView<T> G;
    int rc;
    if ((rc = make_pview<T>(c, p, D, true, false, P, x64, prm->material)) != TB_OK) return rc;
    if ((rc = make_gview<T>(c, g, D, G, m->block_log2)) != TB_OK) return rc;
    if (G.bnum) return fail(c, TB_ERR_UNSUPPORTED, "g2p2g runs on a dense grid");
    BinBuffers B;
    if ((rc = bin_buffers(c, part, P.n, M.nblocks, B)) != TB_OK) return rc;
    if ((rc = touched_buffers(c, M.nblocks)) != TB_OK) return rc;
    const size_t xe = x64 ? sizeof(double) : sizeof(T);
    cudaError_t e = grow(c->g2p2g_x, c->g2p2g_x_cap,
                         std::max<long long>(1, P.n) * D * (long long)xe);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc g2p2g positions");
    const LaunchCfg cfg = cfg_of(c);
    char* xs = c->g2p2g_x;
    PView<T> Pg = P;  // G2P's view: new positions to the scratch, which starts as x
    for (int d = 0; d < D && e == cudaSuccess; ++d) {
        void* dst = xs + size_t(d) * size_t(P.n) * xe;
        const void* src = x64 ? static_cast<const void*>(P.x64[d]) : static_cast<const void*>(P.x[d]);
        e = cudaMemcpyAsync(dst, src, size_t(P.n) * xe, cudaMemcpyDeviceToDevice, c->stream);
        if (x64) Pg.x64_out[d] = static_cast<double*>(dst);
        else Pg.x_out[d] = static_cast<T*>(dst);
    }
    if (e == cudaSuccess) {
        const T* xsrc[3] = {P.x[0], P.x[1], D == 3 ? P.x[2] : P.x[1]};
        const auto M64 = make_dmesh<D, double>(*m);
        const double* xs64[3] = {P.x64[0], P.x64[1], D == 3 ? P.x64[2] : P.x64[1]};
        e = x64 ? launch_bin<D, double>(M64, xs64, P.n, B, cfg) : launch_bin<D, T>(M, xsrc, P.n, B, cfg);
    }
    c->grid_sparse_ok = false;  // dense zero and grid half, as the first step of a call
    if (e == cudaSuccess) e = launch_g2p<D, T, BW>(M, G, Pg, S, B, cfg, false);
    if (e == cudaSuccess) e = p2g_with_zero<D, T, BW>(c, M, P, G, S, B, cfg);
    if (e == cudaSuccess) e = grid_update_sparse_or_dense<D, T, BW>(c, M, G, S, cfg);
    for (int d = 0; d < D && e == cudaSuccess; ++d) {
        void* dst = x64 ? static_cast<void*>(P.x64[d]) : static_cast<void*>(P.x[d]);
        e = cudaMemcpyAsync(dst, xs + size_t(d) * size_t(P.n) * xe, size_t(P.n) * xe, cudaMemcpyDeviceToDevice,
                            c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "g2p2g");
    return TB_OK;
}

template <class T>
int dispatch_g2p2g(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                   const tb_step_params* prm, bool x64) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if ((rc = check_mesh(c, m)) != TB_OK) return rc;
    if ((rc = check_params(c, prm)) != TB_OK) return rc;
    if (prm->transfer != TB_TRANSFER_FLIP)
        return fail(c, TB_ERR_UNSUPPORTED, "g2p2g runs the FLIP/PIC equation set only");
    if (x64 && (prm->basis == TB_WLS_BSPLINE_QUADRATIC || prm->basis == TB_WLS_UGIMP))
        return fail(c, TB_ERR_UNSUPPORTED, "the FP64-position form runs the B-spline / uGIMP step only");
    if (m->dim == 3) return g2p2g_impl<3, T, 4>(c, m, p, part, g, prm, x64);
    if (m->block_log2 == 3) return g2p2g_impl<2, T, 8>(c, m, p, part, g, prm, x64);
    return g2p2g_impl<2, T, 4>(c, m, p, part, g, prm, x64);
}

// ---------------------------------------------------------------------------
// reverse mode
// ---------------------------------------------------------------------------

int check_adjoint_params(tb_ctx* c, const tb_step_params* p) {
    int rc = check_params(c, p);
    if (rc != TB_OK) return rc;
    if (p->material == TB_MATERIAL_VONMISES)
        return fail(c, TB_ERR_UNSUPPORTED, "the adjoint supports the Neo-Hookean and fluid materials only");
    return TB_OK;
}

// The separable, block-scheduled adjoint kernels cover the quadratic B-spline
// and uGIMP with FLIP/PIC; every other basis and APIC take the general
// (particle-parallel, Dual3) reverse step.
bool adjoint_is_general(const tb_step_params* p) {
    return !(p->basis == TB_BSPLINE_QUADRATIC || p->basis == TB_UGIMP) || p->transfer == TB_TRANSFER_APIC;
}

int make_adjview(tb_ctx* c, const tb_adjoint* a, int dim, long long n, AdjView& A, bool apic = false) {
    if (!a) return fail(c, TB_ERR_ARG, "adjoint is NULL");
    std::memset(&A, 0, sizeof A);
    for (int d = 0; d < dim; ++d) {
        A.x[d] = a->x[d];
        A.v[d] = a->v[d];
        if (n && (!A.x[d] || !A.v[d])) return fail(c, TB_ERR_ARG, "adjoint.x/v component %d is NULL", d);
    }
    for (int k = 0; k < dim * dim; ++k) {
        A.F[k] = a->F[k];
        if (n && !A.F[k]) return fail(c, TB_ERR_ARG, "adjoint.F component %d is NULL", k);
    }
    A.mu = a->mu;
    A.lam = a->lambda;
    if (apic)
        for (int k = 0; k < dim * dim; ++k) {
            A.B[k] = a->B[k];
            if (n && !A.B[k]) return fail(c, TB_ERR_ARG, "adjoint.B component %d is NULL (APIC)", k);
        }
    return TB_OK;
}

int grad_grid(tb_ctx* c, int dim, long long nn, GradGrid& GB) {
    const long long need = nn * (1 + 4 * dim);
    cudaError_t e = grow(c->adj_grid, c->adj_grid_cap, need);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc grid sensitivities");
    std::memset(&GB, 0, sizeof GB);
    double* q = c->adj_grid;
    for (int d = 0; d < dim; ++d) GB.vb[d] = q + nn * d;
    q += nn * dim;
    for (int d = 0; d < dim; ++d) GB.vnb[d] = q + nn * d;
    q += nn * dim;
    GB.mb = q;
    q += nn;
    for (int d = 0; d < dim; ++d) GB.pb[d] = q + nn * d;
    q += nn * dim;
    for (int d = 0; d < dim; ++d) GB.fb[d] = q + nn * d;
    return TB_OK;
}

// The three backward kernels for one step. With `recompute` the step's
// partition and forward grid are first rebuilt from `p` into `part` and `g`;
// otherwise `part`, `g` and `totals` (device nactive, nassigned) already hold them.
template <int D, class T, int BW>
int adjoint_impl(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                 const tb_step_params* prm, const tb_adjoint* adj, bool recompute, const int* totals, bool x64) {
    int rc;
    if (recompute) {
        if ((rc = run_step<D, T, BW>(c, m, p, part, g, prm, 1, true, true, true, false, x64)) != TB_OK) return rc;
        totals = c->d_totals;
    }
    const auto M = make_dmesh<D, T>(*m);
    const auto S = make_scalars<T>(*prm);
    PView<T> P;
    GView<T> G;
    AdjView A;
    GradGrid GB;
    const bool apic = prm->transfer == TB_TRANSFER_APIC;
    if ((rc = make_pview<T>(c, p, D, true, apic, P, x64, prm->material)) != TB_OK) return rc;
    if ((rc = make_gview<T>(c, g, D, G, m->block_log2)) != TB_OK) return rc;
    if (G.bnum) return fail(c, TB_ERR_UNSUPPORTED, "the reverse step runs on a dense grid");
    if ((rc = make_adjview(c, adj, D, P.n, A, apic)) != TB_OK) return rc;
    if ((rc = grad_grid(c, D, M.nnodes, GB)) != TB_OK) return rc;
    if (cudaError_t ce = grow(c->adj_coef, c->adj_coef_cap, std::max<long long>(1, P.n) * (2 * D + D * D));
        ce != cudaSuccess)
        return cuda_fail(c, ce, "cudaMalloc scatter coefficients");
    GB.coef = c->adj_coef;
    if (!part || !part->blocklist || !part->offsets || (P.n && (!part->particleindices || !part->blockids)))
        return fail(c, TB_ERR_ARG, "partition array is NULL");
    const AdjPartition AP{totals, part->blocklist, part->offsets, part->particleindices, part->blockids};
    const cudaError_t e = adjoint_is_general(prm) ? launch_adjoint_general<D, T>(M, G, P, S, A, GB, AP, cfg_of(c))
                                                  : launch_adjoint<D, T, BW>(M, G, P, S, A, GB, AP, cfg_of(c));
    return e == cudaSuccess ? TB_OK : cuda_fail(c, e, "adjoint launch");
}

template <class T>
int adjoint_dispatch(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                     const tb_step_params* prm, const tb_adjoint* adj, bool recompute = true,
                     const int* totals = nullptr, bool x64 = false) {
    if (m->dim == 3) return adjoint_impl<3, T, 4>(c, m, p, part, g, prm, adj, recompute, totals, x64);
    if (m->block_log2 == 3) return adjoint_impl<2, T, 8>(c, m, p, part, g, prm, adj, recompute, totals, x64);
    return adjoint_impl<2, T, 4>(c, m, p, part, g, prm, adj, recompute, totals, x64);
}

// The FP64-position form of the reverse step takes the forward form's cases.
int check_x64_adjoint(tb_ctx* c, const tb_mesh* m, const tb_step_params* prm) {
    if (m->dim != 3 && (prm->transfer != TB_TRANSFER_FLIP || prm->basis == TB_WLS_BSPLINE_QUADRATIC ||
                        prm->basis == TB_WLS_UGIMP))
        return fail(c, TB_ERR_UNSUPPORTED, "the FP64-position form runs WLS and APIC in 3D only");
    return TB_OK;
}

template <class T>
int do_adjoint_step(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                    const tb_step_params* prm, const tb_adjoint* adj, bool x64 = false) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK || (rc = check_mesh(c, m)) != TB_OK || (rc = check_adjoint_params(c, prm)) != TB_OK)
        return rc;
    if (x64 && (rc = check_x64_adjoint(c, m, prm)) != TB_OK) return rc;
    if (g && (g->block_numbering || g->active_blocks || g->nactive))
        return fail(c, TB_ERR_UNSUPPORTED, "the reverse step runs on a dense grid");
    return adjoint_dispatch<T>(c, m, p, part, g, prm, adj, true, nullptr, x64);
}

// The state tb_step_* reads and writes, as (particle array, element size)
// fields: x (T, or double in the FP64-position form), v (T), F (double),
// sigma (T), V (T), B (T, APIC). grad_v is output only.
struct StateFields {
    int count = 0;
    void** slot[32];
    size_t elem[32];
};

template <class T>
StateFields state_fields(tb_particles* p, int D, bool apic, bool x64 = false) {
    StateFields f;
    auto add = [&](void** s, size_t e) {
        f.slot[f.count] = s;
        f.elem[f.count] = e;
        ++f.count;
    };
    for (int d = 0; d < D; ++d) add(&p->x[d], x64 ? sizeof(double) : sizeof(T));
    for (int d = 0; d < D; ++d) add(&p->v[d], sizeof(T));
    for (int k = 0; k < D * D; ++k) add(&p->F[k], sizeof(double));
    for (int k = 0; k < (D == 3 ? 6 : 3); ++k) add(&p->sigma[k], sizeof(T));
    add(&p->V, sizeof(T));
    if (apic)
        for (int k = 0; k < D * D; ++k) add(&p->B[k], sizeof(T));
    return f;
}

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

template <class T>
size_t state_bytes(int D, long long n, bool apic, bool x64 = false) {
    const int nf = D + (D == 3 ? 6 : 3) + 1 + (apic ? D * D : 0);  // v, sigma, V, B
    return size_t(nf) * align256(sizeof(T) * size_t(n)) + size_t(D) * align256((x64 ? 8 : sizeof(T)) * size_t(n)) +
           size_t(D * D) * align256(sizeof(double) * size_t(n));
}

// One step of a tape segment: the state before the step, the step's forward
// grid and partition, and its device totals.
template <class T>
size_t slot_bytes(int D, long long n, long long nn, long long nb, bool apic, bool x64 = false) {
    return state_bytes<T>(D, n, apic, x64) + size_t(1 + 4 * D) * align256(sizeof(T) * size_t(nn)) +
           2 * align256(sizeof(int) * size_t(n)) + 2 * align256(sizeof(int) * size_t(nb)) +
           align256(sizeof(int) * size_t(nb + 1)) + 256;
}

template <class T>
void slot_views(char* base, int D, long long n, long long nn, long long nb, bool apic, tb_grid& g,
                tb_partition& part, int*& totals, bool x64 = false) {
    char* q = base + state_bytes<T>(D, n, apic, x64);
    auto take = [&](size_t bytes) {
        char* r = q;
        q += align256(bytes);
        return r;
    };
    g = tb_grid{};
    g.m = take(sizeof(T) * size_t(nn));
    for (int d = 0; d < D; ++d) {
        g.mv[d] = take(sizeof(T) * size_t(nn));
        g.f[d] = take(sizeof(T) * size_t(nn));
        g.v[d] = take(sizeof(T) * size_t(nn));
        g.vn[d] = take(sizeof(T) * size_t(nn));
    }
    part = tb_partition{};
    part.blockids = reinterpret_cast<int32_t*>(take(sizeof(int) * size_t(n)));
    part.particleindices = reinterpret_cast<int32_t*>(take(sizeof(int) * size_t(n)));
    part.counts = reinterpret_cast<int32_t*>(take(sizeof(int) * size_t(nb)));
    part.blocklist = reinterpret_cast<int32_t*>(take(sizeof(int) * size_t(nb)));
    part.offsets = reinterpret_cast<int32_t*>(take(sizeof(int) * size_t(nb + 1)));
    part.nblocks = nb;
    totals = reinterpret_cast<int*>(take(2 * sizeof(int)));
}

// Particles whose state fields point into the snapshot at `base`.
template <class T>
tb_particles snapshot_view(const tb_particles* p, int D, char* base, bool apic, bool x64 = false) {
    tb_particles q = *p;
    StateFields f = state_fields<T>(&q, D, apic, x64);
    size_t off = 0;
    for (int i = 0; i < f.count; ++i) {
        *f.slot[i] = base + off;
        off += align256(f.elem[i] * size_t(p->n));
    }
    return q;
}

template <class T>
int copy_state(tb_ctx* c, const tb_particles* dst, const tb_particles* src, int D, bool apic, bool x64 = false) {
    StateFields fd = state_fields<T>(const_cast<tb_particles*>(dst), D, apic, x64);
    StateFields fs = state_fields<T>(const_cast<tb_particles*>(src), D, apic, x64);
    for (int i = 0; i < fd.count; ++i) {
        if (!*fs.slot[i] || !*fd.slot[i]) return fail(c, TB_ERR_ARG, "particle state field %d is NULL", i);
        const cudaError_t e = cudaMemcpyAsync(*fd.slot[i], *fs.slot[i], fd.elem[i] * size_t(src->n),
                                              cudaMemcpyDeviceToDevice, c->stream);
        if (e != cudaSuccess) return cuda_fail(c, e, "state copy");
    }
    return TB_OK;
}

template <class T>
int do_tape_forward(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                    const tb_step_params* prm, int nsteps, int every, bool x64 = false) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK || (rc = check_mesh(c, m)) != TB_OK || (rc = check_adjoint_params(c, prm)) != TB_OK)
        return rc;
    if (x64 && (rc = check_x64_adjoint(c, m, prm)) != TB_OK) return rc;
    if (nsteps < 0 || every < 1) return fail(c, TB_ERR_ARG, "nsteps must be >= 0 and checkpoint_every >= 1");
    if (!p) return fail(c, TB_ERR_ARG, "particles is NULL");
    const int D = m->dim;
    PView<T> P;
    const bool apic = prm->transfer == TB_TRANSFER_APIC;
    if ((rc = make_pview<T>(c, p, D, true, apic, P, x64, prm->material)) != TB_OK) return rc;
    c->tape_valid = false;
    if (every == 1) {
        // every step kept whole: its input state, grid and partition (the slots
        // the backward pass of a checkpointed tape rebuilds per segment), so the
        // backward pass runs the adjoint kernels only
        long long nn = 1;
        for (int d = 0; d < D; ++d) nn *= m->n_nodes[d];
        const long long nb = mesh_nblocks(m);
        const size_t slot = slot_bytes<T>(D, p->n, nn, nb, apic, x64);
        const long long nslot = std::max(nsteps, 1);
        cudaError_t e = grow(c->tape_cp, c->tape_cp_cap, (long long)(nslot * slot));
        if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc tape");
        for (long long j = 0; j < nslot; ++j) {
            char* base = c->tape_cp + j * slot;
            tb_particles sj = snapshot_view<T>(p, D, base, apic, x64);
            tb_grid gj;
            tb_partition pj;
            int* tj;
            slot_views<T>(base, D, p->n, nn, nb, apic, gj, pj, tj, x64);
            if ((rc = copy_state<T>(c, &sj, p, D, apic, x64)) != TB_OK) return rc;
            if (j >= nsteps) continue;
            if ((rc = dispatch_step<T>(c, m, p, &pj, &gj, prm, 1, true, true, true, true, x64)) != TB_OK) return rc;
            e = cudaMemcpyAsync(tj, c->d_totals, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->stream);
            if (e != cudaSuccess) return cuda_fail(c, e, "tape totals copy");
        }
    } else {
    const long long ncp = nsteps > 0 ? (nsteps + every - 1) / every : 1;
    const size_t sb = state_bytes<T>(D, p->n, apic, x64);
    cudaError_t e = grow(c->tape_cp, c->tape_cp_cap, (long long)(ncp * sb));
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc checkpoints");
    for (long long k = 0; k < ncp; ++k) {
        tb_particles cp = snapshot_view<T>(p, D, c->tape_cp + k * sb, apic, x64);
        if ((rc = copy_state<T>(c, &cp, p, D, apic, x64)) != TB_OK) return rc;
        const int steps = std::min<long long>(every, nsteps - k * every);
        if (steps > 0 && (rc = dispatch_step<T>(c, m, p, part, g, prm, steps, true, true, true, true, x64)) != TB_OK)
            return rc;
    }
    }
    c->tape_valid = true;
    c->tape_n = p->n;
    c->tape_dim = D;
    c->tape_elem = int(sizeof(T));
    c->tape_apic = apic;
    c->tape_x64 = x64;
    c->tape_nsteps = nsteps;
    c->tape_every = every;
    return TB_OK;
}

template <class T>
int do_tape_backward(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                     const tb_step_params* prm, const tb_adjoint* adj, bool x64 = false) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK || (rc = check_mesh(c, m)) != TB_OK || (rc = check_adjoint_params(c, prm)) != TB_OK)
        return rc;
    if (!p) return fail(c, TB_ERR_ARG, "particles is NULL");
    const int D = m->dim;
    const bool apic = prm->transfer == TB_TRANSFER_APIC;
    if (!c->tape_valid || c->tape_n != p->n || c->tape_dim != D || c->tape_elem != int(sizeof(T)) ||
        c->tape_apic != apic || c->tape_x64 != x64)
        return fail(c, TB_ERR_ARG, "no forward tape for these particles on this context (run tb_tape_forward first)");
    (void)part;
    (void)g;
    const int K = c->tape_every, nsteps = c->tape_nsteps;
    long long nn = 1;
    for (int d = 0; d < D; ++d) nn *= m->n_nodes[d];
    const long long nb = mesh_nblocks(m);
    const size_t sb = state_bytes<T>(D, p->n, apic, x64), slot = slot_bytes<T>(D, p->n, nn, nb, apic, x64);
    if (K == 1) {  // the whole tape: the adjoint steps read the slots the forward kept
        for (long long j = nsteps - 1; j >= 0; --j) {
            char* base = c->tape_cp + j * slot;
            tb_particles sj = snapshot_view<T>(p, D, base, apic, x64);
            tb_grid gj;
            tb_partition pj;
            int* tj;
            slot_views<T>(base, D, p->n, nn, nb, apic, gj, pj, tj, x64);
            if ((rc = adjoint_dispatch<T>(c, m, &sj, &pj, &gj, prm, adj, false, tj, x64)) != TB_OK) return rc;
        }
        tb_particles s0 = snapshot_view<T>(p, D, c->tape_cp, apic, x64);
        return copy_state<T>(c, p, &s0, D, apic, x64);
    }
    cudaError_t e = grow(c->tape_seg, c->tape_seg_cap, (long long)(K * slot));
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaMalloc tape segment");
    const long long ncp = nsteps > 0 ? (nsteps + K - 1) / K : 1;
    for (long long k = ncp - 1; k >= 0 && nsteps > 0; --k) {
        const int len = int(std::min<long long>(K, nsteps - k * K));
        tb_particles cp = snapshot_view<T>(p, D, c->tape_cp + k * sb, apic, x64);
        if ((rc = copy_state<T>(c, p, &cp, D, apic, x64)) != TB_OK) return rc;
        // re-run the segment, keeping each step's input state, grid and partition
        for (int j = 0; j < len; ++j) {
            char* base = c->tape_seg + j * slot;
            tb_particles sj = snapshot_view<T>(p, D, base, apic, x64);
            tb_grid gj;
            tb_partition pj;
            int* tj;
            slot_views<T>(base, D, p->n, nn, nb, apic, gj, pj, tj, x64);
            if ((rc = copy_state<T>(c, &sj, p, D, apic, x64)) != TB_OK) return rc;
            if ((rc = dispatch_step<T>(c, m, p, &pj, &gj, prm, 1, true, true, true, j + 1 < len, x64)) != TB_OK) return rc;
            e = cudaMemcpyAsync(tj, c->d_totals, 2 * sizeof(int), cudaMemcpyDeviceToDevice, c->stream);
            if (e != cudaSuccess) return cuda_fail(c, e, "tape totals copy");
        }
        for (int j = len - 1; j >= 0; --j) {
            char* base = c->tape_seg + j * slot;
            tb_particles sj = snapshot_view<T>(p, D, base, apic, x64);
            tb_grid gj;
            tb_partition pj;
            int* tj;
            slot_views<T>(base, D, p->n, nn, nb, apic, gj, pj, tj, x64);
            if ((rc = adjoint_dispatch<T>(c, m, &sj, &pj, &gj, prm, adj, false, tj, x64)) != TB_OK) return rc;
        }
    }
    tb_particles cp0 = snapshot_view<T>(p, D, c->tape_cp, apic, x64);
    return copy_state<T>(c, p, &cp0, D, apic, x64);
}

}  // namespace

extern "C" {

tb_ctx* tb_create(int32_t device, void* stream) {
    tb_ctx* c = new (std::nothrow) tb_ctx();
    if (!c) return nullptr;
    c->device = device;
    c->stream = static_cast<cudaStream_t>(stream);
    if (cudaSetDevice(device) != cudaSuccess) {
        delete c;
        return nullptr;
    }
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
    if (cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess || cudaMalloc(&c->d_totals, 2 * sizeof(int)) != cudaSuccess ||
        cudaMallocHost(&c->h_totals, 2 * sizeof(int)) != cudaSuccess) {
        tb_destroy(c);
        return nullptr;
    }
    cudaMemset(c->d_err, 0, sizeof(int));
    cudaMemset(c->d_totals, 0, 2 * sizeof(int));
    return c;
}

void tb_destroy(tb_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_err);
    cudaFree(c->d_totals);
    if (c->h_totals) cudaFreeHost(c->h_totals);
    cudaFree(c->cursors);
    cudaFree(c->perm_tmp);
    cudaFree(c->partials);
    cudaFree(c->sort_scratch);
    cudaFree(c->roll_buf);
    cudaFree(c->sp_act);
    cudaFree(c->sp_off);
    cudaFree(c->sp_cur);
    cudaFree(c->sp_part);
    cudaFree(c->sp_tot);
    cudaFree(c->touched_cur);
    cudaFree(c->touched_prev);
    cudaFree(c->touched_list);
    cudaFree(c->touched_count);
    cudaFree(c->adj_grid);
    cudaFree(c->adj_coef);
    cudaFree(c->g2p2g_x);
    cudaFree(c->tape_cp);
    cudaFree(c->tape_seg);
    cudaFree(c->ro_scratch);
    cudaFree(c->ro_acc);
    cudaFree(c->wave_max);
    cudaFree(c->ro_decision);
    cudaFree(c->ro_score);
    delete c->prof;
    delete c;
}

const char* tb_last_error(const tb_ctx* c) { return c ? c->error.c_str() : "null context"; }

int32_t tb_set_stream(tb_ctx* c, void* stream) {
    if (!c) return TB_ERR_ARG;
    c->stream = static_cast<cudaStream_t>(stream);
    return TB_OK;
}

int32_t tb_synchronize(tb_ctx* c) {
    int rc = check_ctx(c);
    if (rc != TB_OK) return rc;
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamSynchronize");
    return check_device_status(c);
}

int64_t tb_launch_count(const tb_ctx* c) { return c ? c->launches : 0; }

int32_t tb_profile_enable(tb_ctx* c, int32_t on) {
    int rc = check_ctx(c);
    if (rc != TB_OK) return rc;
    if (on && !c->prof) c->prof = new (std::nothrow) EventProfiler();
    if (on && !c->prof) return fail(c, TB_ERR_ARG, "out of host memory");
    if (!on && c->prof) {
        delete c->prof;
        c->prof = nullptr;
    }
    return TB_OK;
}

int32_t tb_profile_read(tb_ctx* c, tb_kernel_time* out, int32_t cap, int32_t* count) {
    int rc = check_ctx(c);
    if (rc != TB_OK) return rc;
    if (!c->prof) return fail(c, TB_ERR_ARG, "profiling is not enabled");
    if (cap < 0 || (cap > 0 && !out)) return fail(c, TB_ERR_ARG, "bad output buffer");
    c->prof->collect();
    int32_t k = 0;
    for (auto& kv : c->prof->totals) {
        if (k < cap) {
            std::memset(out[k].name, 0, sizeof out[k].name);
            std::strncpy(out[k].name, kv.first.c_str(), sizeof out[k].name - 1);
            out[k].launches = kv.second.first;
            out[k].ms = kv.second.second;
        }
        ++k;
    }
    if (count) *count = k;
    c->prof->totals.clear();
    return TB_OK;
}

int32_t tb_update_weights_f64(tb_ctx* c, const tb_mesh* m, const tb_particles* p, const tb_step_params* prm,
                              tb_weights* w) {
    return do_weights<double>(c, m, p, prm, w);
}
int32_t tb_update_weights_f32(tb_ctx* c, const tb_mesh* m, const tb_particles* p, const tb_step_params* prm,
                              tb_weights* w) {
    return do_weights<float>(c, m, p, prm, w);
}

int32_t tb_update_sparsity_f64(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part, tb_grid* g,
                               int64_t* nstored) {
    return do_update_sparsity<double>(c, m, p, part, g, nstored);
}
int32_t tb_update_sparsity_f32(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part, tb_grid* g,
                               int64_t* nstored) {
    return do_update_sparsity<float>(c, m, p, part, g, nstored);
}
int32_t tb_update_sparsity_f32x64(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part,
                                  tb_grid* g, int64_t* nstored) {
    return do_update_sparsity<float>(c, m, p, part, g, nstored, true);
}
int32_t tb_bin_particles_f64(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part,
                             int64_t* nactive, int64_t* nassigned) {
    return do_bin_only<double>(c, m, p, part, nactive, nassigned);
}
int32_t tb_bin_particles_f32(tb_ctx* c, const tb_mesh* m, const tb_particles* p, tb_partition* part,
                             int64_t* nactive, int64_t* nassigned) {
    return do_bin_only<float>(c, m, p, part, nactive, nassigned);
}

int32_t tb_p2g_f64(tb_ctx* c, const tb_mesh* m, const tb_particles* p, const tb_partition* part, tb_grid* g,
                   const tb_step_params* prm) {
    return dispatch_step<double>(c, m, const_cast<tb_particles*>(p), const_cast<tb_partition*>(part), g, prm, 1,
                                 false, true, false, false);
}
int32_t tb_p2g_f32(tb_ctx* c, const tb_mesh* m, const tb_particles* p, const tb_partition* part, tb_grid* g,
                   const tb_step_params* prm) {
    return dispatch_step<float>(c, m, const_cast<tb_particles*>(p), const_cast<tb_partition*>(part), g, prm, 1,
                                false, true, false, false);
}

int32_t tb_grid_update_f64(tb_ctx* c, const tb_mesh* m, tb_grid* g, const tb_step_params* prm) {
    return do_grid_update<double>(c, m, g, prm);
}
int32_t tb_grid_update_f32(tb_ctx* c, const tb_mesh* m, tb_grid* g, const tb_step_params* prm) {
    return do_grid_update<float>(c, m, g, prm);
}

int32_t tb_g2p_f64(tb_ctx* c, const tb_mesh* m, const tb_grid* g, tb_particles* p, const tb_step_params* prm) {
    return do_g2p_direct<double>(c, m, g, p, prm);
}
int32_t tb_g2p_f32(tb_ctx* c, const tb_mesh* m, const tb_grid* g, tb_particles* p, const tb_step_params* prm) {
    return do_g2p_direct<float>(c, m, g, p, prm);
}

int32_t tb_step_f64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                    const tb_step_params* prm, int32_t nsteps) {
    return dispatch_step<double>(c, m, p, part, g, prm, nsteps, true, true, true, true);
}
int32_t tb_step_f32(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                    const tb_step_params* prm, int32_t nsteps) {
    return dispatch_step<float>(c, m, p, part, g, prm, nsteps, true, true, true, true);
}

int32_t tb_step_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                       const tb_step_params* prm, int32_t nsteps) {
    return dispatch_step<float>(c, m, p, part, g, prm, nsteps, true, true, true, true, true);
}

int32_t tb_g2p2g_f64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                     const tb_step_params* prm) {
    return dispatch_g2p2g<double>(c, m, p, part, g, prm, false);
}
int32_t tb_g2p2g_f32(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                     const tb_step_params* prm) {
    return dispatch_g2p2g<float>(c, m, p, part, g, prm, false);
}
int32_t tb_g2p2g_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                        const tb_step_params* prm) {
    return dispatch_g2p2g<float>(c, m, p, part, g, prm, true);
}

int32_t tb_step_reorder_f64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                            const tb_step_params* prm, int32_t nsteps, double threshold) {
    return dispatch_step<double>(c, m, p, part, g, prm, nsteps, true, true, true, true, false, threshold);
}
int32_t tb_step_reorder_f32(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                            const tb_step_params* prm, int32_t nsteps, double threshold) {
    return dispatch_step<float>(c, m, p, part, g, prm, nsteps, true, true, true, true, false, threshold);
}
int32_t tb_step_reorder_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                               const tb_step_params* prm, int32_t nsteps, double threshold) {
    return dispatch_step<float>(c, m, p, part, g, prm, nsteps, true, true, true, true, true, threshold);
}

int32_t tb_reorder_particles_f64(tb_ctx* c, int32_t dim, tb_particles* p, tb_partition* part, double threshold,
                                 int32_t* reordered) {
    return do_reorder(c, p, part, dim, sizeof(double), false, threshold, reordered, nullptr);
}
int32_t tb_reorder_particles_f32(tb_ctx* c, int32_t dim, tb_particles* p, tb_partition* part, double threshold,
                                 int32_t* reordered) {
    return do_reorder(c, p, part, dim, sizeof(float), false, threshold, reordered, nullptr);
}
int32_t tb_reorder_particles_f32x64(tb_ctx* c, int32_t dim, tb_particles* p, tb_partition* part, double threshold,
                                    int32_t* reordered) {
    return do_reorder(c, p, part, dim, sizeof(float), true, threshold, reordered, nullptr);
}

int32_t tb_particle_contiguity(tb_ctx* c, const tb_partition* part, int64_t n, double* score) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    if (!score) return fail(c, TB_ERR_ARG, "score is NULL");
    if (n < 0 || n > 0x7fffffffll) return fail(c, TB_ERR_CAPACITY, "particle count exceeds Int32 capacity");
    ReorderArgs RA{};
    if ((rc = reorder_args(c, const_cast<tb_partition*>(part), n, 0.0, RA)) != TB_OK) return rc;
    RA.report_outside = false;
    cudaError_t e = launch_reorder_score(RA, cfg_of(c));
    double sc = 1.0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&sc, c->ro_score, sizeof sc, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "contiguity");
    *score = sc;
    return TB_OK;
}

int32_t tb_max_wave_speed_f64(tb_ctx* c, int32_t dim, const tb_particles* p, const tb_step_params* prm,
                              double* c_max) {
    return do_wave_speed<double>(c, dim, p, prm, c_max);
}
int32_t tb_max_wave_speed_f32(tb_ctx* c, int32_t dim, const tb_particles* p, const tb_step_params* prm,
                              double* c_max) {
    return do_wave_speed<float>(c, dim, p, prm, c_max);
}

int32_t tb_rollout_host_f64(tb_ctx* c, const tb_mesh* m, tb_particles* host, const tb_step_params* prm,
                            int32_t nsteps) {
    return do_rollout<double>(c, m, host, prm, nsteps);
}
int32_t tb_rollout_host_f32(tb_ctx* c, const tb_mesh* m, tb_particles* host, const tb_step_params* prm,
                            int32_t nsteps) {
    return do_rollout<float>(c, m, host, prm, nsteps);
}

int32_t tb_rollout_host_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* host, const tb_step_params* prm,
                               int32_t nsteps) {
    return do_rollout<float>(c, m, host, prm, nsteps, true);
}

int32_t tb_adjoint_step_f64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                            const tb_step_params* prm, tb_adjoint* adj) {
    return do_adjoint_step<double>(c, m, p, part, g, prm, adj);
}
int32_t tb_adjoint_step_f32(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                            const tb_step_params* prm, tb_adjoint* adj) {
    return do_adjoint_step<float>(c, m, p, part, g, prm, adj);
}
int32_t tb_adjoint_step_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                               const tb_step_params* prm, tb_adjoint* adj) {
    return do_adjoint_step<float>(c, m, p, part, g, prm, adj, true);
}

int32_t tb_tape_forward_f64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                            const tb_step_params* prm, int32_t nsteps, int32_t every) {
    return do_tape_forward<double>(c, m, p, part, g, prm, nsteps, every);
}
int32_t tb_tape_forward_f32(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                            const tb_step_params* prm, int32_t nsteps, int32_t every) {
    return do_tape_forward<float>(c, m, p, part, g, prm, nsteps, every);
}
int32_t tb_tape_backward_f64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                             const tb_step_params* prm, tb_adjoint* adj) {
    return do_tape_backward<double>(c, m, p, part, g, prm, adj);
}
int32_t tb_tape_backward_f32(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                             const tb_step_params* prm, tb_adjoint* adj) {
    return do_tape_backward<float>(c, m, p, part, g, prm, adj);
}
int32_t tb_tape_forward_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                               const tb_step_params* prm, int32_t nsteps, int32_t every) {
    return do_tape_forward<float>(c, m, p, part, g, prm, nsteps, every, true);
}
int32_t tb_tape_backward_f32x64(tb_ctx* c, const tb_mesh* m, tb_particles* p, tb_partition* part, tb_grid* g,
                                const tb_step_params* prm, tb_adjoint* adj) {
    return do_tape_backward<float>(c, m, p, part, g, prm, adj, true);
}

int64_t tb_tape_bytes(const tb_mesh* m, int64_t n, int32_t elem, int32_t apic, int32_t x64, int32_t nsteps,
                      int32_t checkpoint_every) {
    if (!m || (m->dim != 2 && m->dim != 3) || n < 0 || (elem != 4 && elem != 8) || nsteps < 0 ||
        checkpoint_every < 1)
        return -1;
    const int D = m->dim;
    long long nn = 1;
    for (int d = 0; d < D; ++d) {
        if (m->n_nodes[d] < 1) return -1;
        nn *= m->n_nodes[d];
    }
    const long long nb = mesh_nblocks(m);
    const bool ap = apic != 0, xd = x64 != 0 && elem == 4;
    const size_t sb = elem == 4 ? state_bytes<float>(D, n, ap, xd) : state_bytes<double>(D, n, ap);
    const size_t slot = elem == 4 ? slot_bytes<float>(D, n, nn, nb, ap, xd) : slot_bytes<double>(D, n, nn, nb, ap);
    if (checkpoint_every == 1) return (int64_t)(std::max(nsteps, 1) * slot);
    const long long ncp = nsteps > 0 ? (nsteps + checkpoint_every - 1) / checkpoint_every : 1;
    return (int64_t)(ncp * sb + (long long)checkpoint_every * slot);
}

int32_t tb_tape_release(tb_ctx* c) {
    int rc;
    if ((rc = check_ctx(c)) != TB_OK) return rc;
    const cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamSynchronize");
    cudaFree(c->tape_cp);
    cudaFree(c->tape_seg);
    c->tape_cp = c->tape_seg = nullptr;
    c->tape_cp_cap = c->tape_seg_cap = 0;
    c->tape_valid = false;
    return TB_OK;
}

}  // extern "C"
