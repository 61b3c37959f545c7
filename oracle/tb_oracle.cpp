// tb_oracle.cpp -- extern "C" entry points of the CPU oracle (libtb_oracle.so).
//
// TEST INFRASTRUCTURE ONLY: loaded by tests/, __graft_entry__.smoke() and the
// CPU legs of bench.py through ctypes. Never linked into libtesserae_b200.so.
//
// prec: 0 = FP64 (all double), 1 = mixed FP32 (float state, double F).
#include "tb_oracle.hpp"

#include <omp.h>

using namespace tbo;

namespace {

template <int D, class T>
int do_bin(const tb_mesh* m, const tb_particles* p, tb_partition* part, int64_t* na, int64_t* nass) {
    auto M = make_mesh<D, T>(*m);
    if (part->nblocks != M.nblocks) return TB_ERR_ARG;
    bin<D, T>(M, *p, *part, na, nass);
    return TB_OK;
}

template <int D, class T>
int do_weights(const tb_mesh* m, const tb_particles* p, const tb_step_params* prm, tb_weights* wt) {
    auto M = make_mesh<D, T>(*m);
    constexpr int NW = nwin<D>();
    for (int64_t i = 0; i < p->n; ++i) {
        T x[3] = {0, 0, 0};
        for (int d = 0; d < D; ++d) x[d] = CP<T>(p->x[d])[i];
        Weights<D, T> W;
        compute_weights(M, prm->basis, x, opt<T>(p->l, i, prm->gimp_l), W);
        for (int s = 0; s < NW; ++s) {
            P<T>(wt->w)[i * NW + s] = W.w[s];
            for (int d = 0; d < D; ++d) P<T>(wt->grad_w)[(i * NW + s) * D + d] = W.dw[s][d];
        }
        for (int d = 0; d < D; ++d) {
            if (W.empty) {
                wt->window[i * 2 * D + 2 * d] = 1;
                wt->window[i * 2 * D + 2 * d + 1] = 0;
            } else {
                wt->window[i * 2 * D + 2 * d] = W.lo[d] + 1;
                wt->window[i * 2 * D + 2 * d + 1] = W.lo[d] + W.cnt[d];
            }
        }
    }
    return TB_OK;
}

template <int D, class T>
int do_p2g(const tb_mesh* m, const tb_particles* p, tb_grid* g, const tb_step_params* prm) {
    auto M = make_mesh<D, T>(*m);
    p2g<D, T>(M, *p, *g, *prm);
    return TB_OK;
}

template <int D, class T>
int do_grid(const tb_mesh* m, tb_grid* g, const tb_step_params* prm) {
    auto M = make_mesh<D, T>(*m);
    grid_update<D, T>(M, *g, *prm);
    return TB_OK;
}

template <int D, class T>
int do_g2p(const tb_mesh* m, const tb_grid* g, tb_particles* p, const tb_step_params* prm) {
    auto M = make_mesh<D, T>(*m);
    g2p<D, T>(M, *g, *p, *prm);
    return TB_OK;
}

// Sequential reference step: P2G in particle order, dense grid update, G2P.
template <int D, class T>
int do_step(const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm, int nsteps) {
    auto M = make_mesh<D, T>(*m);
    for (int s = 0; s < nsteps; ++s) {
        p2g<D, T>(M, *p, *g, *prm);
        grid_update<D, T>(M, *g, *prm);
        g2p<D, T>(M, *g, *p, *prm);
    }
    return TB_OK;
}

// @G2P2G (src/Transfer/g2p2g.jl:98-159) for the FLIP/PIC equation set: one
// pass over the particles, each doing its G2P and then its P2G with the weights
// bound to the position it had before the G2P half moved it (g2p2g.jl:103-106);
// the P2G half reads the updated v, sigma and V. Its assigned targets m, mv, f
// are zeroed first, and the grid half of README.md:75-76 runs after the pass
// (G2P2G_halves, g2p2g.jl:14-18).
template <int D, class T>
int do_g2p2g(const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm) {
    if (prm->transfer != TB_TRANSFER_FLIP) return TB_ERR_UNSUPPORTED;
    auto M = make_mesh<D, T>(*m);
    zero_p2g_targets(M, *g);
    T* gmv[3] = {nullptr, nullptr, nullptr};
    T* gf[3] = {nullptr, nullptr, nullptr};
    for (int d = 0; d < D; ++d) {
        gmv[d] = P<T>(g->mv[d]);
        gf[d] = P<T>(g->f[d]);
    }
    for (int64_t i = 0; i < p->n; ++i) {
        T x0[3] = {T(0), T(0), T(0)};
        for (int d = 0; d < D; ++d) x0[d] = CP<T>(p->x[d])[i];
        g2p_particle<D, T>(M, *g, *p, *prm, i);
        ParticleIn<D, T> q;
        load_particle<D, T>(*p, *prm, i, q);
        for (int d = 0; d < D; ++d) q.x[d] = x0[d];
        p2g_particle<D, T, void>(M, *prm, q, P<T>(g->m), gmv, gf);
    }
    grid_update<D, T>(M, *g, *prm);
    return TB_OK;
}

// Multithreaded step following the reference CPU path: partition update with
// per-thread histograms (cpu_block_strategy.jl:89-190), colour-phased block
// scatter (region.jl:212-256), parallel grid half and parallel G2P
// (threads.jl:25-53). Per-phase seconds are accumulated into `phase_s[4]`
// (bin, p2g, grid, g2p) when non-null.
template <int D, class T>
int do_step_parallel(const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm, int nsteps,
                     int nthreads, double* phase_s) {
    auto M = make_mesh<D, T>(*m);
    const int64_t n = p->n, nb = M.nblocks;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int nt = 1;
#pragma omp parallel
    {
#pragma omp single
        nt = omp_get_num_threads();
    }
    std::vector<int32_t> blockid(n), perm(n), offsets(nb + 1);
    std::vector<int32_t> hist(size_t(nt) * size_t(nb));
    std::vector<std::vector<int32_t>> colour_blocks(1 << D);
    T* gmv[3] = {nullptr, nullptr, nullptr};
    T* gf[3] = {nullptr, nullptr, nullptr};
    for (int d = 0; d < D; ++d) { gmv[d] = P<T>(g->mv[d]); gf[d] = P<T>(g->f[d]); }

    for (int s = 0; s < nsteps; ++s) {
        double t0 = omp_get_wtime();
        // ---- partition: per-thread histograms over contiguous chunks, stable scatter
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel
        {
            int t = omp_get_thread_num();
            int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
            int32_t* h = hist.data() + size_t(t) * nb;
            for (int64_t i = lo; i < hi; ++i) {
                T x[3] = {0, 0, 0};
                for (int d = 0; d < D; ++d) x[d] = CP<T>(p->x[d])[i];
                int32_t b = findblock(M, x);
                blockid[i] = b;
                if (b) h[b - 1]++;
            }
        }
        int64_t acc = 0;
        for (auto& cb : colour_blocks) cb.clear();
        for (int64_t b = 0; b < nb; ++b) {
            offsets[b] = int32_t(acc);
            int64_t cnt = 0;
            for (int t = 0; t < nt; ++t) {
                int32_t c = hist[size_t(t) * nb + b];
                hist[size_t(t) * nb + b] = int32_t(acc + cnt);
                cnt += c;
            }
            if (cnt) colour_blocks[block_colour(M, b)].push_back(int32_t(b));
            acc += cnt;
        }
        offsets[nb] = int32_t(acc);
#pragma omp parallel
        {
            int t = omp_get_thread_num();
            int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
            int32_t* h = hist.data() + size_t(t) * nb;
            for (int64_t i = lo; i < hi; ++i) {
                int32_t b = blockid[i];
                if (b) perm[h[b - 1]++] = int32_t(i);
            }
        }
        double t1 = omp_get_wtime();
        // ---- P2G: zero the assigned targets, then colour phases
#pragma omp parallel for schedule(static)
        for (int64_t I = 0; I < M.nnodes; ++I) {
            P<T>(g->m)[I] = T(0);
            for (int d = 0; d < D; ++d) { gmv[d][I] = T(0); gf[d][I] = T(0); }
        }
        for (int c = 0; c < (1 << D); ++c) {
            const auto& cb = colour_blocks[c];
#pragma omp parallel for schedule(dynamic, 4)
            for (int64_t k = 0; k < int64_t(cb.size()); ++k) {
                int32_t b = cb[k];
                for (int32_t j = offsets[b]; j < offsets[b + 1]; ++j) {
                    ParticleIn<D, T> q;
                    load_particle<D, T>(*p, *prm, perm[j], q);
                    p2g_particle<D, T, void>(M, *prm, q, P<T>(g->m), gmv, gf);
                }
            }
        }
        double t2 = omp_get_wtime();
#pragma omp parallel for schedule(static)
        for (int64_t I = 0; I < M.nnodes; ++I) grid_update_node(M, *g, *prm, I);
        double t3 = omp_get_wtime();
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) g2p_particle(M, *g, *p, *prm, i);
        double t4 = omp_get_wtime();
        if (phase_s) {
            phase_s[0] += t1 - t0;
            phase_s[1] += t2 - t1;
            phase_s[2] += t3 - t2;
            phase_s[3] += t4 - t3;
        }
    }
    return TB_OK;
}

// One step backwards (reverse mode of do_step's step; no reference counterpart).
template <int D, class T>
int do_adjoint_step(const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm, tb_adjoint* a) {
    auto M = make_mesh<D, T>(*m);
    if (adjoint_supported(*prm)) return adjoint_step<D, T>(M, *p, *g, *prm, *a);
    // WLS and KernelCorrection bases, APIC: the general reverse step
    return adjoint_step_general<D, T>(*m, M, *p, *g, *prm, *a);
}

#define TBO_DISPATCH(FN, ...)                                                   \
    do {                                                                        \
        if (m == nullptr) return TB_ERR_ARG;                                    \
        if (m->dim == 3 && prec == 0) return FN<3, double>(__VA_ARGS__);        \
        if (m->dim == 3 && prec == 1) return FN<3, float>(__VA_ARGS__);         \
        if (m->dim == 2 && prec == 0) return FN<2, double>(__VA_ARGS__);        \
        if (m->dim == 2 && prec == 1) return FN<2, float>(__VA_ARGS__);         \
        return TB_ERR_UNSUPPORTED;                                              \
    } while (0)

}  // namespace

extern "C" {

int tbo_bin(int prec, const tb_mesh* m, const tb_particles* p, tb_partition* part, int64_t* na, int64_t* nass) {
    TBO_DISPATCH(do_bin, m, p, part, na, nass);
}

int tbo_update_weights(int prec, const tb_mesh* m, const tb_particles* p, const tb_step_params* prm,
                       tb_weights* w) {
    TBO_DISPATCH(do_weights, m, p, prm, w);
}

int tbo_p2g(int prec, const tb_mesh* m, const tb_particles* p, tb_grid* g, const tb_step_params* prm) {
    TBO_DISPATCH(do_p2g, m, p, g, prm);
}

int tbo_grid_update(int prec, const tb_mesh* m, tb_grid* g, const tb_step_params* prm) {
    TBO_DISPATCH(do_grid, m, g, prm);
}

int tbo_g2p(int prec, const tb_mesh* m, const tb_grid* g, tb_particles* p, const tb_step_params* prm) {
    TBO_DISPATCH(do_g2p, m, g, p, prm);
}

int tbo_g2p2g(int prec, const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm) {
    TBO_DISPATCH(do_g2p2g, m, p, g, prm);
}

int tbo_step(int prec, const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm, int nsteps) {
    TBO_DISPATCH(do_step, m, p, g, prm, nsteps);
}

int tbo_step_parallel(int prec, const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm,
                      int nsteps, int nthreads, double* phase_s) {
    TBO_DISPATCH(do_step_parallel, m, p, g, prm, nsteps, nthreads, phase_s);
}

int tbo_adjoint_step(int prec, const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm,
                     tb_adjoint* a) {
    TBO_DISPATCH(do_adjoint_step, m, p, g, prm, a);
}

// The sequential step in forward-mode dual numbers: every particle and grid
// array (F included) holds (value, derivative) pairs of doubles.
int tbo_step_dual(const tb_mesh* m, tb_particles* p, tb_grid* g, const tb_step_params* prm, int nsteps) {
    if (m == nullptr) return TB_ERR_ARG;
    if (prm->material == TB_MATERIAL_VONMISES) return TB_ERR_UNSUPPORTED;
    if (m->dim == 3) return do_step<3, Dual>(m, p, g, prm, nsteps);
    if (m->dim == 2) return do_step<2, Dual>(m, p, g, prm, nsteps);
    return TB_ERR_UNSUPPORTED;
}

int tbo_max_threads(void) { return omp_get_max_threads(); }

// 1-D jets for the known-answer tests of test/basis.jl:309-311.
void tbo_jet_bspline_quadratic(double xi, double* val, double* der) { jet_bspline_quadratic(xi, *val, *der); }
void tbo_jet_ugimp(double xi, double l, double* val, double* der) { jet_ugimp(xi, l, *val, *der); }

// Support window of one point (1-based inclusive start/stop per axis).
int tbo_supportnodes(int prec, const tb_mesh* m, int basis, const double* x, double l, int64_t* out) {
    if (!m || m->dim < 2 || m->dim > 3) return TB_ERR_ARG;
    if (m->dim == 3 && prec == 0) {
        auto M = make_mesh<3, double>(*m);
        Weights<3, double> W;
        compute_weights(M, basis, x, l, W);
        for (int d = 0; d < 3; ++d) {
            out[2 * d] = W.empty ? 1 : W.lo[d] + 1;
            out[2 * d + 1] = W.empty ? 0 : W.lo[d] + W.cnt[d];
        }
        return TB_OK;
    }
    if (m->dim == 2 && prec == 0) {
        auto M = make_mesh<2, double>(*m);
        Weights<2, double> W;
        compute_weights(M, basis, x, l, W);
        for (int d = 0; d < 2; ++d) {
            out[2 * d] = W.empty ? 1 : W.lo[d] + 1;
            out[2 * d + 1] = W.empty ? 0 : W.lo[d] + W.cnt[d];
        }
        return TB_OK;
    }
    return TB_ERR_UNSUPPORTED;
}

}  // extern "C"
