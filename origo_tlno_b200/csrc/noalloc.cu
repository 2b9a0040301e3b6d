// tlno_gpu_eri_blocks_noalloc: the ERI-block endpoint without any device
// allocation, for callers that cannot call cudaMalloc / cudaFree -- code that
// runs under a strict device-memory budget owned by another allocator (a
// framework memory pool that must not be fragmented or bypassed), code on a
// latency-critical path where an allocation may synchronise the device, or
// code that must not grow the device footprint after start-up.
//
// The per-call scratch of the ERI-block kernel (the ad-hoc shell-pair table,
// the primitive-pair records and the class-sorted quartet lists) lives in
// one file-scope device array of kNoAllocScratchBytes.  Every device on which
// a context is created holds that array until process exit: context creation
// looks up its device address (cudaGetSymbolAddress, with that device
// current), which also loads this file's device code under lazy module
// loading, so the 8 MiB are taken then and never by the entry point itself.
// A call on a device without a context looks the address up itself and
// should therefore come before any stream capture.  All calls share the one array,
// so calls whose work overlaps on the GPU (for instance two contexts driven
// from two host threads) race on it.  A call rewrites every scratch byte it
// reads before the kernels read it, so nothing left by an earlier call has to
// be cleared.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "context.hpp"
#include "kernels.hpp"
#include "launch_types.hpp"
#include "plan.hpp"

namespace {

constexpr std::size_t kNoAllocScratchBytes = 8u << 20;  // 8 MiB

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device, resolved once.
void* scratch_address(int device) {
    static std::mutex mtx;
    static void* addr[256] = {nullptr};
    if (device < 0 || device >= 256) throw tlno_gpu::Error(TLNO_GPU_E_INVALID, "tlno_gpu: invalid device index");
    std::lock_guard<std::mutex> lock(mtx);
    if (!addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            throw tlno_gpu::Error(TLNO_GPU_E_CUDA, std::string("tlno_gpu: scratch symbol lookup failed: ") +
                                                       cudaGetErrorString(e));
        addr[device] = p;
    }
    return addr[device];
}

std::size_t align256(std::size_t n) { return (n + 255) & ~static_cast<std::size_t>(255); }

}  // namespace

void tlno_gpu::noalloc_prepare(int device) { (void)scratch_address(device); }

extern "C" int tlno_gpu_eri_blocks_noalloc(tlno_gpu_context* ctx, int n_quartets, const int* shells4,
                                           const long long* offsets, double* d_out) {
    using namespace tlno_gpu;
    try {
        if (!ctx || n_quartets < 0 || (n_quartets > 0 && (!shells4 || !offsets || !d_out)))
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        unsigned char* scratch = static_cast<unsigned char*>(scratch_address(ctx->device));
        if (n_quartets == 0) return TLNO_GPU_OK;
        const Basis& b = ctx->basis;
        const int ns = static_cast<int>(b.shells.size());
        // Host staging of the tables (host memory only).
        std::vector<int> pA, pB, pnp, poff;
        std::vector<dev::DPrimPair> prim;
        std::vector<std::vector<int>> by_class(625);
        for (int q = 0; q < n_quartets; ++q) {
            const int* sh = shells4 + 4 * q;
            for (int k = 0; k < 4; ++k)
                if (sh[k] < 0 || sh[k] >= ns) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: shell index out of range");
            if (offsets[q] < 0) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: negative output offset");
            for (int side = 0; side < 2; ++side) {
                pA.push_back(sh[2 * side]);
                pB.push_back(sh[2 * side + 1]);
                poff.push_back(static_cast<int>(prim.size()));
                const std::size_t before = prim.size();
                primitive_pairs(b, sh[2 * side], sh[2 * side + 1], prim);
                pnp.push_back(static_cast<int>(prim.size() - before));
            }
            const int la = b.shells[sh[0]].L, lb = b.shells[sh[1]].L, lc = b.shells[sh[2]].L, ld = b.shells[sh[3]].L;
            by_class[((la * 5 + lb) * 5 + lc) * 5 + ld].push_back(q);
        }
        std::vector<int> qb, qk, cls_begin, cls_key;
        std::vector<long long> oo;
        for (int key = 0; key < 625; ++key) {
            if (by_class[key].empty()) continue;
            cls_begin.push_back(static_cast<int>(qb.size()));
            cls_key.push_back(key);
            for (int q : by_class[key]) {
                qb.push_back(2 * q);
                qk.push_back(2 * q + 1);
                oo.push_back(offsets[q]);
            }
        }
        cls_begin.push_back(static_cast<int>(qb.size()));
        // Scratch layout, 256-byte aligned sections.
        const std::size_t np = pA.size();
        std::size_t off = 0;
        const std::size_t o_A = off;    off += align256(np * sizeof(int));
        const std::size_t o_B = off;    off += align256(np * sizeof(int));
        const std::size_t o_np = off;   off += align256(np * sizeof(int));
        const std::size_t o_off = off;  off += align256(np * sizeof(int));
        const std::size_t o_prim = off; off += align256(prim.size() * sizeof(dev::DPrimPair));
        const std::size_t o_qb = off;   off += align256(qb.size() * sizeof(int));
        const std::size_t o_qk = off;   off += align256(qk.size() * sizeof(int));
        const std::size_t o_oo = off;   off += align256(oo.size() * sizeof(long long));
        if (off > kNoAllocScratchBytes)
            throw Error(TLNO_GPU_E_INVALID,
                        "tlno_gpu_eri_blocks_noalloc: the request needs " + std::to_string(off) +
                            " bytes of scratch; the fixed scratch holds " + std::to_string(kNoAllocScratchBytes) +
                            " bytes -- split the quartets into smaller calls");
        std::vector<unsigned char> stage(off, 0);
        std::memcpy(stage.data() + o_A, pA.data(), np * sizeof(int));
        std::memcpy(stage.data() + o_B, pB.data(), np * sizeof(int));
        std::memcpy(stage.data() + o_np, pnp.data(), np * sizeof(int));
        std::memcpy(stage.data() + o_off, poff.data(), np * sizeof(int));
        if (!prim.empty()) std::memcpy(stage.data() + o_prim, prim.data(), prim.size() * sizeof(dev::DPrimPair));
        std::memcpy(stage.data() + o_qb, qb.data(), qb.size() * sizeof(int));
        std::memcpy(stage.data() + o_qk, qk.data(), qk.size() * sizeof(int));
        std::memcpy(stage.data() + o_oo, oo.data(), oo.size() * sizeof(long long));
        cudaStream_t s = ctx->stream;
        TLNO_CUDA(cudaMemcpyAsync(scratch, stage.data(), off, cudaMemcpyHostToDevice, s));
        dev::PlanView pv{};
        pv.shell_xyz = ctx->d_shell_xyz.as<double>();
        pv.shell_L = ctx->d_shell_L.as<int>();
        pv.shell_sph = ctx->d_shell_sph.as<int>();
        pv.pair_A = reinterpret_cast<const int*>(scratch + o_A);
        pv.pair_B = reinterpret_cast<const int*>(scratch + o_B);
        pv.pair_nprim = reinterpret_cast<const int*>(scratch + o_np);
        pv.pair_prim_off = reinterpret_cast<const int*>(scratch + o_off);
        pv.prim = reinterpret_cast<const dev::DPrimPair*>(scratch + o_prim);
        for (std::size_t c = 0; c + 1 < cls_begin.size(); ++c) {
            const int key = cls_key[c];
            dev::ClassLaunch cl{};
            cl.la = key / 125;
            cl.lb = (key / 25) % 5;
            cl.lc = (key / 5) % 5;
            cl.ld = key % 5;
            cl.q_bra = reinterpret_cast<const int*>(scratch + o_qb) + cls_begin[c];
            cl.q_ket = reinterpret_cast<const int*>(scratch + o_qk) + cls_begin[c];
            cl.out_off = reinterpret_cast<const long long*>(scratch + o_oo) + cls_begin[c];
            cl.n_quartets = cls_begin[c + 1] - cls_begin[c];
            cl.out = d_out;
            launch_eri_store(pv, cl, s);
        }
        // The host staging buffer must outlive the copy.
        TLNO_CUDA(cudaStreamSynchronize(s));
        return TLNO_GPU_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return TLNO_GPU_E_INVALID;
    }
}
