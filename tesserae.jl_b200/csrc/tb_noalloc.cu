// tb_noalloc.cu -- particle binning that allocates nothing.
//
// tb_bin_particles_noalloc bins particles exactly like tb_bin_particles_f32/f64
// (same kernels, same bit-exact output), for callers that cannot call
// cudaMalloc: code running inside another framework's memory pool or a host
// runtime that forbids device allocation after start-up, real-time loops that
// must never stall on the allocator, and callers without a tb_ctx. Instead of
// context-owned buffers it uses one fixed scratch array compiled into this
// library as a file-scope __device__ variable, so the only device memory it
// touches besides the caller's arrays is that array, which every GPU that loads
// the library holds until the process exits.
//
// Limits: at most TB_NOALLOC_MAX_PARTICLES particles and TB_NOALLOC_MAX_BLOCKS
// grid blocks per call (24 MiB of scratch); larger inputs are rejected with
// TB_ERR_CAPACITY. All calls share the one array: calls that overlap on the GPU
// (two streams, or two host threads) race and corrupt each other's result, so
// serialise them. The array keeps the previous call's contents; every scratch
// word a call reads is written earlier in the same call, so nothing is cleared.
#include <cstdio>

#include "tb_launch.cuh"

namespace {

constexpr long long kMaxParticles = 1ll << 20;
constexpr long long kMaxBlocks = 1ll << 20;
constexpr long long kTiles = (kMaxBlocks + tb::SCAN_TILE - 1) / tb::SCAN_TILE;

// Byte offsets of the pieces of the scratch array (each 256-byte aligned).
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kOffCursors = 0;
constexpr size_t kOffPermTmp = kOffCursors + align256(sizeof(int) * kMaxBlocks);
constexpr size_t kOffPartials = kOffPermTmp + align256(sizeof(int) * kMaxParticles);
constexpr size_t kOffSort = kOffPartials + align256(sizeof(unsigned long long) * kTiles);
constexpr size_t kOffTotals = kOffSort + align256(sizeof(unsigned long long) * 2 * kMaxParticles);
constexpr size_t kBytes = kOffTotals + 256;

__device__ __align__(256) unsigned char tb_noalloc_scratch[kBytes];

void report(char* errbuf, int32_t errlen, const char* msg) {
    if (errbuf && errlen > 0) std::snprintf(errbuf, size_t(errlen), "%s", msg);
}

// Device address of the scratch array on the current device. In host code the
// symbol names a host-side stand-in, so the address is looked up with the
// device current. It is looked up on every call, not cached: after
// cudaDeviceReset (or any teardown of the primary context) the module is
// loaded again and the array can move. Once the module is loaded the lookup
// allocates nothing; the first call on a device may load the module (lazy
// loading), which is when the driver reserves the array.
int scratch_address(void** out, char* errbuf, int32_t errlen) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, tb_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "tb_bin_particles_noalloc: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
        report(errbuf, errlen, msg);
        return TB_ERR_CUDA;
    }
    *out = p;
    return TB_OK;
}

template <int D, class T>
int run(const tb_mesh* m, const tb_particles* p, tb_partition* part, cudaStream_t stream, long long nb,
        unsigned char* scratch, int64_t* nactive, int64_t* nassigned, char* errbuf, int32_t errlen) {
    const tb::DMesh<D, T> M = tb::make_dmesh<D, T>(*m);
    const T* xs[3] = {static_cast<const T*>(p->x[0]), static_cast<const T*>(p->x[1]),
                      static_cast<const T*>(p->x[D == 3 ? 2 : 1])};
    tb::BinBuffers B;
    B.blockids = part->blockids;
    B.counts = part->counts;
    B.offsets = part->offsets;
    B.blocklist = part->blocklist;
    B.perm = part->particleindices;
    B.cursors = reinterpret_cast<int*>(scratch + kOffCursors);
    B.perm_tmp = reinterpret_cast<int*>(scratch + kOffPermTmp);
    B.partials = reinterpret_cast<unsigned long long*>(scratch + kOffPartials);
    B.sort_scratch = reinterpret_cast<unsigned long long*>(scratch + kOffSort);
    B.totals = reinterpret_cast<int*>(scratch + kOffTotals);
    int device = 0;
    cudaGetDevice(&device);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    long long launches = 0;
    const tb::LaunchCfg cfg{stream, sms, &launches, nullptr, nullptr};
    cudaError_t e = tb::launch_bin<D, T>(M, xs, p->n, B, cfg);
    int h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, B.totals, sizeof h, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        char msg[256];
        std::snprintf(msg, sizeof msg, "tb_bin_particles_noalloc: %s", cudaGetErrorString(e));
        report(errbuf, errlen, msg);
        return TB_ERR_CUDA;
    }
    (void)nb;
    if (nactive) *nactive = h[0];
    if (nassigned) *nassigned = h[1];
    return TB_OK;
}

}  // namespace

extern "C" int32_t tb_bin_particles_noalloc(const tb_mesh* mesh, const tb_particles* particles, int32_t precision,
                                            tb_partition* partition, void* stream, int64_t* nactive,
                                            int64_t* nassigned, char* errbuf, int32_t errlen) {
    if (!mesh || !particles || !partition) {
        report(errbuf, errlen, "tb_bin_particles_noalloc: NULL mesh, particles or partition");
        return TB_ERR_ARG;
    }
    if (precision != 0 && precision != 1) {
        report(errbuf, errlen, "tb_bin_particles_noalloc: precision must be 0 (double) or 1 (float)");
        return TB_ERR_ARG;
    }
    const int dim = mesh->dim;
    if (!((dim == 3 && mesh->block_log2 == 2) || (dim == 2 && (mesh->block_log2 == 2 || mesh->block_log2 == 3)))) {
        report(errbuf, errlen, "tb_bin_particles_noalloc: supported meshes are 3D with block_log2 2, 2D with 2 or 3");
        return TB_ERR_UNSUPPORTED;
    }
    long long nb = 1;
    for (int d = 0; d < dim; ++d) {
        if (mesh->n_nodes[d] < 2) {
            report(errbuf, errlen, "tb_bin_particles_noalloc: every mesh axis needs at least 2 nodes");
            return TB_ERR_ARG;
        }
        nb *= ((mesh->n_nodes[d] - 1) >> mesh->block_log2) + 1;
    }
    const long long n = particles->n;
    if (n < 0 || n > kMaxParticles || nb > kMaxBlocks) {
        char msg[256];
        std::snprintf(msg, sizeof msg,
                      "tb_bin_particles_noalloc: %lld particles / %lld blocks exceed the fixed scratch limit of "
                      "%lld particles / %lld blocks; use tb_bin_particles_f32/_f64",
                      n, nb, kMaxParticles, kMaxBlocks);
        report(errbuf, errlen, msg);
        return TB_ERR_CAPACITY;
    }
    if (partition->nblocks != nb) {
        report(errbuf, errlen, "tb_bin_particles_noalloc: partition.nblocks does not match the mesh");
        return TB_ERR_ARG;
    }
    if (!partition->counts || !partition->offsets || !partition->blocklist ||
        (n && (!partition->blockids || !partition->particleindices))) {
        report(errbuf, errlen, "tb_bin_particles_noalloc: NULL partition array");
        return TB_ERR_ARG;
    }
    for (int d = 0; d < dim; ++d)
        if (n && !particles->x[d]) {
            report(errbuf, errlen, "tb_bin_particles_noalloc: NULL particle position array");
            return TB_ERR_ARG;
        }
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) {
        report(errbuf, errlen, "tb_bin_particles_noalloc: no current CUDA device");
        return TB_ERR_CUDA;
    }
    void* scratch = nullptr;
    const int rc = scratch_address(&scratch, errbuf, errlen);
    if (rc != TB_OK) return rc;
    unsigned char* s = static_cast<unsigned char*>(scratch);
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dim == 3)
        return precision ? run<3, float>(mesh, particles, partition, st, nb, s, nactive, nassigned, errbuf, errlen)
                         : run<3, double>(mesh, particles, partition, st, nb, s, nactive, nassigned, errbuf, errlen);
    return precision ? run<2, float>(mesh, particles, partition, st, nb, s, nactive, nassigned, errbuf, errlen)
                     : run<2, double>(mesh, particles, partition, st, nb, s, nactive, nassigned, errbuf, errlen);
}
