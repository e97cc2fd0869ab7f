// FP64 matrix product C = A B^T on the int8 tensor cores of sm_100a (tcgen05.mma kind::i8), for
// the line of sight's frequency sum theta[k, l] = sum_q A[k, q] B[l, q] (cmb.py:809-834), whose
// FP64 form is one DGEMM.  The digit splitting is described in dgemm_i8.cuh.
//
// Pipeline (one stream, no host synchronisation):
//   1. row_scale_kernel: per row of A and of B the power-of-two scale 2^e > max|x| * 128/127
//   2. slice_kernel: the digit planes d_s (int8) written in the tensor cores' shared-memory
//      order (8-row x 16-byte core matrices, K-major, no swizzle), one contiguous 32 KB block
//      per (plane, 256-row tile, 128-byte K stage), so one bulk copy moves a stage
//   3. gemm_kernel: one CTA per (256-row tile of A, 256-row tile of B, K range); warp 0 streams
//      the stages of every digit pair with cp.async.bulk into a 3-deep shared-memory ring,
//      warp 1 issues the MMAs (two M = 128, N = 256, K = 32 instructions per 32-byte K step,
//      accumulators in TMEM: 2 x 256 columns of int32), warps 2-5 read each level's exact int32
//      sums with tcgen05.ld and store them (write-only, so a level boundary costs the tensor
//      cores one TMEM drain, not a read-modify-write of FP64 partials in DRAM)
//   4. reduce_kernel: C = the scaled sum over levels and K ranges
// Every wait on a barrier is bounded in time; a CTA whose wait runs out sets the error flag,
// lets its issued copies and MMAs finish, frees its TMEM and returns, and the reduction then
// writes NaN into C.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "discoeb.h"
#include "dgemm_i8.cuh"

namespace dgemm_i8 {
namespace {

constexpr int BM = 256;               // rows of A per tile: two M = 128 MMAs
constexpr int BN = 256;               // rows of B per tile: the MMA's N
constexpr int BKB = 128;              // K bytes (int8 elements) per pipeline stage
constexpr int STAGES = 3;
constexpr int TILE = 256 * BKB;       // bytes of one operand's stage (32 KB)
constexpr int THREADS = 192;          // warp 0 loads, warp 1 issues MMAs, warps 2-5 drain TMEM
constexpr int SMEM_BYTES = 2 * STAGES * TILE + 1024 + 256;
constexpr uint64_t kWaitNs = 4000000000ull;  // a barrier wait gives up after 4 s

struct Geo {
    int m, n, k, slices, split;
    int mt, nt, kst;
    size_t err, ea, eb, sa, sb, da, db, part, total;
    size_t a_plane, b_plane;  // bytes of one digit plane
    long long ldp;            // row pitch of the level sums (int32)
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

int sm_count()
{
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                  cudaSuccess || sms <= 0) {
        cudaGetLastError();
        return 148;
    }
    return sms;
}

// K ranges per tile: the smallest count (<= 4, <= the K stages) giving at least four waves of
// CTAs (one per SM), so that the last, partial wave is a small part of the work; more ranges
// add level sums to store and reduce
int choose_split(int units, int kst, int sms)
{
    int s = 1;
    while (s < 4 && s < kst && (long long)units * s < 4LL * sms) ++s;
    return s;
}

bool geometry(int m, int n, int k, int slices, int split, Geo& g)
{
    if (m < 1 || n < 1 || k < 1 || slices < 1 || slices > kMaxSlices) return false;
    g.m = m;
    g.n = n;
    g.k = k;
    g.slices = slices;
    g.mt = (m + BM - 1) / BM;
    g.nt = (n + BN - 1) / BN;
    g.kst = (k + BKB - 1) / BKB;
    if (split <= 0) split = choose_split(g.mt * g.nt, g.kst, sm_count());
    g.split = std::max(1, std::min(split, g.kst));
    g.a_plane = (size_t)g.mt * g.kst * TILE;
    g.b_plane = (size_t)g.nt * g.kst * TILE;
    g.ldp = (long long)g.nt * BN;
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t at = o; o = align256(o + bytes); return at; };
    g.err = take(sizeof(int));
    g.ea = take(sizeof(int) * (size_t)g.mt * BM);
    g.eb = take(sizeof(int) * (size_t)g.nt * BN);
    g.sa = take(sizeof(double) * (size_t)g.mt * BM);
    g.sb = take(sizeof(double) * (size_t)g.nt * BN);
    g.da = take(g.a_plane * slices);
    g.db = take(g.b_plane * slices);
    g.part = take(sizeof(int) * (size_t)g.split * slices * g.mt * BM * g.ldp);
    g.total = o;
    return true;
}

// ---- PTX wrappers ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the completion of the barrier phase of this parity.  False when another role of the
// CTA has given up (abort != nullptr and set) or after kWaitNs.
__device__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int* abort)
{
    const uint64_t t0 = globaltimer();
    for (uint32_t i = 0; i < 0x7fffffffu; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255u) == 255u) {
            if (abort && *abort) return false;
            if (globaltimer() - t0 > kWaitNs) return false;
        }
    }
    return false;
}

__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; lbo = bytes between the two 16-byte K
// chunks of an instruction, sbo = bytes between 8-row groups; version 1 (bits 46-47)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}

// tcgen05.wait::ld with the loaded registers as operands, so that no use is scheduled before it
__device__ __forceinline__ void tmem_wait_ld(uint32_t (&r)[32])
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

// ---- splitting ------------------------------------------------------------------------------

// One block per (padded) row: e = the exponent of 2^e > max_k |x| * 128/127, so that the first
// digit x 2^(7-e) rounds into [-127, 127]; scale = 2^(e-7) (NaN for a row holding a non-finite
// value, which then makes its products NaN; 0 digits for it and for padding rows).
__global__ void row_scale_kernel(int rows, int k, const double* __restrict__ X, long long ld, int* __restrict__ e,
                                 double* __restrict__ scale)
{
    __shared__ double red[32];
    const int r = blockIdx.x;
    double mx = 0.0;
    bool finite = true;
    if (r < rows) {
        const double* row = X + (size_t)r * ld;
        for (int j = threadIdx.x; j < k; j += blockDim.x) {
            const double a = fabs(row[j]);
            finite = finite && isfinite(a);
            mx = fmax(mx, a);
        }
    }
    const bool all_finite = __syncthreads_and(finite);
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, red[w]);
        int ex = 0;
        if (all_finite && mx > 0.0) frexp(mx * (128.0 / 127.0) * (1.0 + 0x1p-40), &ex);
        e[r] = all_finite ? ex : 0;
        scale[r] = all_finite ? (mx > 0.0 ? ldexp(1.0, ex - 7) : 0.0) : __longlong_as_double(0x7ff8000000000000ll);
    }
}

// The same for a transposed operand (element (r, j) at X[j * ld + r]): a block per 32 rows, lane =
// row, the 8 warps striding over K, so every load instruction reads 32 consecutive doubles
__global__ void row_scale_t_kernel(int rows, int rows_pad, int k, const double* __restrict__ X, long long ld,
                                   int* __restrict__ e, double* __restrict__ scale)
{
    __shared__ double red[8][32];
    __shared__ int bad[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int r = blockIdx.x * 32 + lane;
    double mx = 0.0;
    int nonfinite = 0;
    if (r < rows)
        for (int j = w; j < k; j += 8) {
            const double a = fabs(X[(size_t)j * ld + r]);
            nonfinite |= !isfinite(a);
            mx = fmax(mx, a);
        }
    red[w][lane] = mx;
    bad[w][lane] = nonfinite;
    __syncthreads();
    if (w == 0 && r < rows_pad) {
        for (int i = 1; i < 8; ++i) {
            mx = fmax(mx, red[i][lane]);
            nonfinite |= bad[i][lane];
        }
        int ex = 0;
        if (!nonfinite && mx > 0.0) frexp(mx * (128.0 / 127.0) * (1.0 + 0x1p-40), &ex);
        e[r] = nonfinite ? 0 : ex;
        scale[r] = nonfinite ? __longlong_as_double(0x7ff8000000000000ll) : (mx > 0.0 ? ldexp(1.0, ex - 7) : 0.0);
    }
}

// One thread per (padded row, 16 consecutive K elements): its `slices` digits, each plane's 16
// bytes stored at the row's place in the 8 x 16-byte core matrix of its stage block.  Thread
// order = (row within the core matrix, 16-byte chunk, 8-row group, stage, tile), so a warp writes
// 512 contiguous bytes per plane.
// (element (r, j) at X[r * ld + j], or at X[j * ld + r] for a transposed operand).
__global__ void slice_kernel(int rows, int k, const double* __restrict__ X, long long ld, bool trans,
                             const int* __restrict__ e, const double* __restrict__ scale, int kst, long long n_units,
                             int slices, size_t plane, uint8_t* __restrict__ D)
{
    const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_units) return;
    const int rr = (int)(u & 7), c = (int)((u >> 3) & 7), g = (int)((u >> 6) & 31);
    const long long rest = u >> 11;
    const int kc = (int)(rest % kst);
    const long long rb = rest / kst;
    const long long row = rb * 256 + g * 8 + rr;
    const long long k0 = (long long)kc * BKB + c * 16;
    double x[16];
    const bool live = row < rows && isfinite(scale[row]) && scale[row] != 0.0;
    const int sh = 7 - (live ? e[row] : 0);
#pragma unroll
    for (int j = 0; j < 16; ++j)
        x[j] = (live && k0 + j < k) ? ldexp(trans ? X[(size_t)(k0 + j) * ld + row] : X[(size_t)row * ld + k0 + j], sh)
                                    : 0.0;
    uint8_t* dst = D + ((size_t)rb * kst + kc) * TILE + g * 1024 + c * 128 + rr * 16;
    for (int s = 0; s < slices; ++s) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const double d = rint(x[j]);
            x[j] = (x[j] - d) * 128.0;
            w[j >> 2] |= ((uint32_t)(int)d & 0xffu) << (8 * (j & 3));
        }
        *reinterpret_cast<uint4*>(dst + (size_t)s * plane) = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

// ---- the tensor-core product ----------------------------------------------------------------

__global__ void __launch_bounds__(THREADS, 1)
    gemm_kernel(int mt_count, int nt_count, int kst, int split, int slices, size_t a_plane, size_t b_plane,
                const uint8_t* __restrict__ DA, const uint8_t* __restrict__ DB, int* __restrict__ levels,
                long long ldp, int* __restrict__ err)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    uint8_t* sa = smem;
    uint8_t* sb = smem + STAGES * TILE;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * STAGES * TILE);  // full, empty, accfull, accempty, fin
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 2 * STAGES + 3);
    volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);
    auto full = [&](int i) { return smem_u32(bars + i); };
    auto empty = [&](int i) { return smem_u32(bars + STAGES + i); };
    const uint32_t accfull = smem_u32(bars + 2 * STAGES), accempty = smem_u32(bars + 2 * STAGES + 1),
                   fin = smem_u32(bars + 2 * STAGES + 2);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mt = blockIdx.x % mt_count;
    const int nt = (blockIdx.x / mt_count) % nt_count;
    const int sp = blockIdx.x / (mt_count * nt_count);
    const int st0 = (int)((long long)sp * kst / split), st1 = (int)((long long)(sp + 1) * kst / split);

    if (threadIdx.x == 0) {
        for (int i = 0; i < STAGES; ++i) {
            mbar_init(full(i), 1);
            mbar_init(empty(i), 1);
        }
        mbar_init(accfull, 1);
        mbar_init(accempty, 4);
        mbar_init(fin, 1);
        *abort = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;

    if (warp == 0 && lane == 0) {
        // producer: every (level, digit pair, stage) in the order the MMA warp consumes them
        long long it = 0;
        bool ok = true;
        for (int lev = 0; lev < slices && ok; ++lev)
            for (int s = 0; s <= lev && ok; ++s) {
                const uint8_t* pa = DA + (size_t)s * a_plane + (size_t)mt * kst * TILE;
                const uint8_t* pb = DB + (size_t)(lev - s) * b_plane + (size_t)nt * kst * TILE;
                for (int st = st0; st < st1; ++st, ++it) {
                    const int slot = (int)(it % STAGES);
                    const long long use = it / STAGES;
                    if (use > 0 && !mbar_wait(empty(slot), (uint32_t)((use - 1) & 1), abort)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(full(slot), 2 * TILE);
                    bulk_load(smem_u32(sa + slot * TILE), pa + (size_t)st * TILE, TILE, full(slot));
                    bulk_load(smem_u32(sb + slot * TILE), pb + (size_t)st * TILE, TILE, full(slot));
                }
            }
        if (!ok) {
            *abort = 1;
            atomicExch(err, 1);
        }
        // every issued copy has landed before the CTA may exit
        for (int slot = 0; slot < STAGES; ++slot) {
            const long long uses = (it - slot + STAGES - 1) / STAGES;
            if (uses > 0 && !mbar_wait(full(slot), (uint32_t)((uses - 1) & 1), nullptr)) atomicExch(err, 1);
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: level by level, the digit pairs (s, lev - s) accumulate into the same two
        // TMEM accumulators (rows 0-127 and 128-255 of the tile), exact in int32
        const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                               ((uint32_t)(128 >> 4) << 24);
        long long it = 0;
        bool ok = true;
        for (int lev = 0; lev < slices && ok; ++lev) {
            if (lev > 0 && !mbar_wait(accempty, (uint32_t)((lev - 1) & 1), abort)) {
                ok = false;
                break;
            }
            tc_fence_after();
            bool first = true;
            for (int s = 0; s <= lev && ok; ++s)
                for (int st = st0; st < st1; ++st, ++it) {
                    const int slot = (int)(it % STAGES);
                    const long long use = it / STAGES;
                    if (!mbar_wait(full(slot), (uint32_t)(use & 1), abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t a0 = smem_u32(sa + slot * TILE), b0 = smem_u32(sb + slot * TILE);
#pragma unroll
                    for (int q = 0; q < BKB / 32; ++q) {
                        const uint64_t bd = smem_desc(b0 + q * 256, 128, 1024);
                        mma_i8(tbase, smem_desc(a0 + q * 256, 128, 1024), bd, idesc, (first && q == 0) ? 0u : 1u);
                        mma_i8(tbase + 256, smem_desc(a0 + 16384 + q * 256, 128, 1024), bd, idesc,
                               (first && q == 0) ? 0u : 1u);
                    }
                    first = false;
                    mma_commit(empty(slot));
                }
            if (ok) mma_commit(accfull);
        }
        if (!ok) {
            *abort = 1;
            atomicExch(err, 1);
        }
        // every issued MMA has completed before TMEM is released
        mma_commit(fin);
        if (!mbar_wait(fin, 0, nullptr)) atomicExch(err, 1);
    } else if (warp >= 2) {
        // TMEM drain: warp w reads TMEM lanes 32 (w % 4) .. + 31, i.e. one tile row per thread
        const int quarter = warp & 3;
        const int lrow = quarter * 32 + lane;
        for (int lev = 0; lev < slices; ++lev) {
            int ok = 0;
            if (lane == 0) ok = mbar_wait(accfull, (uint32_t)(lev & 1), abort) ? 1 : 0;
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) {
                if (lane == 0) {
                    *abort = 1;
                    atomicExch(err, 1);
                }
                break;
            }
            tc_fence_after();
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const long long row = (long long)mt * BM + h * 128 + lrow;
                int* orow = levels + (((size_t)sp * slices + lev) * mt_count * BM + row) * ldp + (size_t)nt * BN;
#pragma unroll 1
                for (int c0 = 0; c0 < BN; c0 += 32) {
                    uint32_t r[32];
                    tmem_ld32(tbase + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(h * 256 + c0), r);
                    tmem_wait_ld(r);
                    uint4* o4 = reinterpret_cast<uint4*>(orow + c0);
#pragma unroll
                    for (int j = 0; j < 8; ++j) o4[j] = make_uint4(r[4 * j], r[4 * j + 1], r[4 * j + 2], r[4 * j + 3]);
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(accempty);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tbase) : "memory");
    }
}

// C[i, j] = 2^(eA_i - 7) 2^(eB_j - 7) sum over the K ranges and levels of 128^-level times the
// level's exact int32 sum (smallest weights first); NaN everywhere when a kernel gave up
__global__ void reduce_kernel(int m, int n, int split, int slices, const int* __restrict__ levels, long long ldp,
                              long long plane, const double* __restrict__ SA, const double* __restrict__ SB,
                              const int* __restrict__ err, double* __restrict__ C, long long ldc)
{
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)m * n) return;
    const long long i = idx / n, j = idx % n;
    double v = 0.0;
    for (int lev = slices - 1; lev >= 0; --lev) {
        long long acc = 0;
        for (int s = 0; s < split; ++s) acc += levels[((long long)s * slices + lev) * plane + i * ldp + j];
        v = v * 0.0078125 + (double)acc;  // Horner in 1/128: exact scaling, one rounding per level
    }
    v = (v * SB[j]) * SA[i];
    C[i * ldc + j] = *err ? __longlong_as_double(0x7ff8000000000000ll) : v;
}

std::mutex g_attr_mu;
bool g_attr_set[64] = {};

}  // namespace

int64_t workspace_bytes(int m, int n, int k, int slices, int split)
{
    Geo g;
    if (!geometry(m, n, k, slices, split, g)) return -1;
    return (int64_t)g.total;
}

int32_t run(int m, int n, int k, const double* A, int64_t lda, bool trans_a, const double* B, int64_t ldb,
            bool trans_b, double* C, int64_t ldc, int slices, int split, char* ws, int64_t ws_bytes, void* stream)
{
    Geo g;
    if (!geometry(m, n, k, slices, split, g) || !A || !B || !C || !ws || lda < (trans_a ? m : k) ||
        ldb < (trans_b ? n : k) || ldc < n)
        return DISCOEB_EINVAL;
    if (ws_bytes < (int64_t)g.total || (reinterpret_cast<uintptr_t>(ws) & 255u)) return DISCOEB_EINVAL;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DISCOEB_ECUDA;
    {
        std::lock_guard<std::mutex> lock(g_attr_mu);
        if (!g_attr_set[dev]) {
            if (cudaFuncSetAttribute(gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES) !=
                cudaSuccess)
                return DISCOEB_ECUDA;
            g_attr_set[dev] = true;
        }
    }
    int* err = reinterpret_cast<int*>(ws + g.err);
    int* ea = reinterpret_cast<int*>(ws + g.ea);
    int* eb = reinterpret_cast<int*>(ws + g.eb);
    double* sa = reinterpret_cast<double*>(ws + g.sa);
    double* sb = reinterpret_cast<double*>(ws + g.sb);
    uint8_t* da = reinterpret_cast<uint8_t*>(ws + g.da);
    uint8_t* db = reinterpret_cast<uint8_t*>(ws + g.db);
    int* levels = reinterpret_cast<int*>(ws + g.part);
    cudaMemsetAsync(err, 0, sizeof(int), s);
    if (trans_a)
        row_scale_t_kernel<<<g.mt * BM / 32, 256, 0, s>>>(m, g.mt * BM, k, A, lda, ea, sa);
    else
        row_scale_kernel<<<g.mt * BM, 256, 0, s>>>(m, k, A, lda, ea, sa);
    if (trans_b)
        row_scale_t_kernel<<<g.nt * BN / 32, 256, 0, s>>>(n, g.nt * BN, k, B, ldb, eb, sb);
    else
        row_scale_kernel<<<g.nt * BN, 256, 0, s>>>(n, k, B, ldb, eb, sb);
    const long long ua = (long long)g.mt * BM * g.kst * (BKB / 16), ub = (long long)g.nt * BN * g.kst * (BKB / 16);
    slice_kernel<<<(unsigned)((ua + 255) / 256), 256, 0, s>>>(m, k, A, lda, trans_a, ea, sa, g.kst, ua, slices,
                                                              g.a_plane, da);
    slice_kernel<<<(unsigned)((ub + 255) / 256), 256, 0, s>>>(n, k, B, ldb, trans_b, eb, sb, g.kst, ub, slices,
                                                              g.b_plane, db);
    gemm_kernel<<<(unsigned)(g.mt * g.nt * g.split), THREADS, SMEM_BYTES, s>>>(
        g.mt, g.nt, g.kst, g.split, slices, g.a_plane, g.b_plane, da, db, levels, g.ldp, err);
    const long long mn = (long long)m * n;
    reduce_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(m, n, g.split, slices, levels, g.ldp,
                                                               (long long)g.mt * BM * g.ldp, sa, sb, err, C, ldc);
    return cudaGetLastError() == cudaSuccess ? DISCOEB_SUCCESS : DISCOEB_ECUDA;
}

}  // namespace dgemm_i8

extern "C" {

int64_t discoeb_dgemm_i8_workspace_bytes(int32_t m, int32_t n, int32_t k, int32_t slices, int32_t split)
{
    return dgemm_i8::workspace_bytes(m, n, k, slices, split);
}

int32_t discoeb_dgemm_i8(int32_t m, int32_t n, int32_t k, const double* A, int64_t lda, int32_t trans_a,
                         const double* B, int64_t ldb, int32_t trans_b, double* C, int64_t ldc, int32_t slices,
                         int32_t split, void* workspace, int64_t workspace_bytes, void* stream)
{
    if ((trans_a != 0 && trans_a != 1) || (trans_b != 0 && trans_b != 1)) return DISCOEB_EINVAL;
    return dgemm_i8::run(m, n, k, A, lda, trans_a != 0, B, ldb, trans_b != 0, C, ldc, slices, split,
                         static_cast<char*>(workspace), workspace_bytes, stream);
}

}  // extern "C"
