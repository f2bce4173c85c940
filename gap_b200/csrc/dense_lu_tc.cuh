// Dense-tail LU with the trailing update on the 5th-generation tensor cores (tcgen05).
//
// Same right-looking factorisation, without pivoting, as k_dense_lu (one CTA per scenario, FP32,
// panels of W = 32 columns; steps A and B unchanged: warp 0 factors the diagonal block in
// registers, every thread solves whole rows of L21 and columns of U12), but step C -- the rank-32
// update A22 -= L21 U12 -- runs as tcgen05.mma kind::tf32 on 128 x 128 tiles with the accumulator
// in tensor memory:
//   * operands: the tile's 128 rows of L21 (K-major, read from the factor's rows) and 128
//     columns of U12 (read from the panel's rows), each split into a TF32 high part (rounded to
//     nearest) and the FP32 remainder, staged in shared memory in the canonical K-major layout
//     without swizzle (8-row x 16-byte core matrices; leading byte offset = one 4-element K chunk
//     of all rows, stride byte offset = 128 bytes);
//   * D^T = Uhi^T Lhi^T + Ulo^T Lhi^T + Uhi^T Llo^T (3 x 4 instructions of K = 8, issued by one
//     thread, their completion signalled to an mbarrier with tcgen05.commit; the transposed
//     product puts one tile column in each tensor-memory lane) -- FP32-level accuracy (the
//     dropped lo x lo term is below 2^-21 of the product);
//   * tiles go column block by column block: U12 is staged once per block and L21 once per
//     tile, each thread writing whole 16-byte K chunks of 32 consecutive rows or columns per warp
//     (no shared-memory bank conflicts);
//   * epilogue: each thread owns one tile column (its warp's tensor-memory lane quarter) and
//     half of its rows, so every load and store of a warp covers 32 adjacent columns of a row;
//     the first 32 of its 64 C values are loaded while the MMAs run, then C - D is written back
//     straight from the tcgen05.ld registers, and the next tile's operands are staged.
// Shared memory is 64 KB of operands plus the panel's L11 / U11 / 1/diag and 128 registers per
// thread, so two CTAs share an SM, holding 128 tensor-memory columns each (with the split
// path's k_dlu_update_tc beside them, shared memory and registers still keep the columns in use
// below the SM's 512): the allocation never waits.  Every wait on the mbarrier is bounded: when
// one runs out (the CTA agrees on it with a barrier), the kernel waits once more, bounded, for
// the MMAs in flight, marks the scenario singular, sets ctrl[5], frees its tensor memory and
// ends.  The bound is 200 ms of %globaltimer time (tc_wait).
#pragma once

#include <cstdint>

namespace gapk {

constexpr int TC_M = 128, TC_N = 128, TC_W = 32;
// operand buffers: A hi, A lo, B hi, B lo, each TC_M (or TC_N) rows x TC_W values
constexpr int TC_OPER_BYTES = 4 * TC_M * TC_W * 4;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Byte offset of element (r, k) of a rows x TC_W operand in the K-major, no-swizzle layout.
__device__ __forceinline__ int tc_kmaj(int r, int k, int rows) {
    return (k >> 2) * (rows / 8) * 128 + (r >> 3) * 128 + (r & 7) * 16 + (k & 3) * 4;
}
// Shared-memory matrix descriptor (no swizzle): start, leading / stride byte offsets, version 1.
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((addr >> 4) & 0x3FFF) |
           (static_cast<uint64_t>((lbo >> 4) & 0x3FFF) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// TF32 high part (round to nearest) and the FP32 remainder.
__device__ __forceinline__ void tc_split(float x, float& hi, float& lo) {
    uint32_t u;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(u) : "f"(x));
    hi = __uint_as_float(u);
    lo = x - hi;
}
// Wait for the mbarrier phase `phase` to complete, for at most TC_WAIT_NS of %globaltimer time
// (and at most 2^24 polls): false when the bound ran out.  A tile's MMAs take about a
// microsecond; the bound leaves room for the context being time-sliced with others.
constexpr unsigned long long TC_WAIT_NS = 200000000ull;
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t phase) {
    unsigned long long t0 = 0;  // read only once a wait lasts (a normal one ends within 64 polls)
    for (int it = 0; it < (1 << 24); ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(phase)
            : "memory");
        if (done) return true;
        if ((it & 63) == 63) {
            const unsigned long long t = gtimer();
            if (it == 63) t0 = t;
            else if (t - t0 > TC_WAIT_NS) return false;
        }
    }
    return false;
}
// 16 consecutive tensor-memory columns of this thread's lane.
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int c = 0; c < 16; ++c) v[c] = __uint_as_float(r[c]);
}

// Stage A = the L21 rows row0.. of one 128-row tile (global rows k0 + W + row0 + r, columns
// k0..k0 + W - 1), split into hi / lo.  Thread e of the CTA takes row r = e % 128 and the K
// chunk e / 128, so the 32 lanes of a warp store 32 consecutive rows of one chunk: 512
// contiguous bytes of the core-matrix layout (no bank conflict).  Rows past n2 are zero.
__device__ __forceinline__ void tc_stage_a(const float* __restrict__ Am, int ld, int k0, int n2,
                                           int row0, unsigned char* oper) {
    unsigned char* Ah = oper;
    unsigned char* Al = oper + TC_M * TC_W * 4;
#pragma unroll
    for (int i = 0; i < TC_M * (TC_W / 4) / 256; ++i) {
        const int e = threadIdx.x + 256 * i;
        const int r = e & (TC_M - 1), k4 = (e / TC_M) * 4;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (row0 + r < n2)
            v = *reinterpret_cast<const float4*>(Am + (size_t)(k0 + TC_W + row0 + r) * ld + k0 + k4);
        float4 h, l;
        tc_split(v.x, h.x, l.x);
        tc_split(v.y, h.y, l.y);
        tc_split(v.z, h.z, l.z);
        tc_split(v.w, h.w, l.w);
        const int o = tc_kmaj(r, k4, TC_M);
        *reinterpret_cast<float4*>(Ah + o) = h;
        *reinterpret_cast<float4*>(Al + o) = l;
    }
}

// Stage B = the U12 columns col0.. of one 128-column block (global rows k0..k0 + W - 1, columns
// k0 + W + col0 + n), split into hi / lo.  Thread e takes column n = e % 128 and the K chunk
// e / 128: four loads down the column (a warp reads 128 consecutive bytes of each row) and one
// 16-byte store of the chunk, the lanes' stores contiguous.  Columns past n2 are zero.
__device__ __forceinline__ void tc_stage_b(const float* __restrict__ Am, int ld, int k0, int n2,
                                           int col0, unsigned char* oper) {
    unsigned char* Bh = oper + 2 * TC_M * TC_W * 4;
    unsigned char* Bl = oper + 2 * TC_M * TC_W * 4 + TC_N * TC_W * 4;
#pragma unroll
    for (int i = 0; i < TC_N * (TC_W / 4) / 256; ++i) {
        const int e = threadIdx.x + 256 * i;
        const int n = e & (TC_N - 1), k4 = (e / TC_N) * 4;
        float x[4] = {0.f, 0.f, 0.f, 0.f};
        if (col0 + n < n2) {
            const float* c = Am + (size_t)(k0 + k4) * ld + k0 + TC_W + col0 + n;
#pragma unroll
            for (int t = 0; t < 4; ++t) x[t] = c[(size_t)t * ld];
        }
        float4 h, l;
        tc_split(x[0], h.x, l.x);
        tc_split(x[1], h.y, l.y);
        tc_split(x[2], h.z, l.z);
        tc_split(x[3], h.w, l.w);
        const int o = tc_kmaj(n, k4, TC_N);
        *reinterpret_cast<float4*>(Bh + o) = h;
        *reinterpret_cast<float4*>(Bl + o) = l;
    }
}

// One CTA per scenario (256 threads).  Float, W = 32.  Dynamic shared memory: TC_OPER_BYTES
// (operands; the no-swizzle layout needs 16-byte alignment only) + U11^T, L11 [W][W + 4] and
// 1/diag [W].
__global__ void __launch_bounds__(256, 2) k_dense_lu_tc(BatchDev B, int N) {
    constexpr int W = TC_W;
    const int q = blockIdx.x;
    if (q >= B.n_scen || !B.solving[q] || (B.gfactor && !B.gfactor[q / B.sw])) return;
    const int ld = dense_ld(N);
    float* A = reinterpret_cast<float*>(B.Dt) + (size_t)q * N * ld;
    const bool wait_test = B.ctrl[6] != 0;  // test hook: issue no MMAs (the waits run out)
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* oper = smraw;
    float* U11 = reinterpret_cast<float*>(smraw + TC_OPER_BYTES);  // [W][W + 4] transposed
    float* SL = U11 + W * (W + 4);                                 // [W][W + 4] L11 row-major
    float* SD = SL + W * (W + 4);                                  // [W] 1 / diag(U11)
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tslot;
    __shared__ int bad, timed_out;
    const int tid = threadIdx.x, nt = blockDim.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tslot)),
                     "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        bad = 0;
        timed_out = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = tslot;
    uint32_t phase = 0;
    // F32 accumulate, TF32 A and B, both K-major, N = 128, M = 128
    const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);
    constexpr uint32_t LBO_A = (TC_M / 8) * 128, LBO_B = (TC_N / 8) * 128;
    auto stamp = [&](int j, bool copy_prev) {
        if (B.dlu_ts && tid == 0) {
            unsigned long long* t = B.dlu_ts + (size_t)q * (1 + 3 * ((N + W - 1) / W)) + j;
            *t = copy_prev ? t[-1] : gtimer();
        }
    };
    stamp(0, false);
    for (int k0 = 0; k0 < N && !timed_out; k0 += W) {
        const int w = min(W, N - k0);
        const int m = N - k0;
        const int n2 = m - w;
        // ---- A: diagonal block, warp 0
        if (tid < 32) {
            if (dense_diag_block<float, W>(A, ld, k0, w, U11, W + 4, SL, SD)) bad = 1;
        }
        __syncthreads();
        stamp(1 + 3 * (k0 / W), false);
        if (n2 > 0) {
            // ---- B: rows of L21 and columns of U12
            for (int it = tid; it < 2 * n2; it += nt) {
                if (it < n2)
                    dense_l21_row<float, W>(A + (size_t)(k0 + W + it) * ld + k0, U11, W + 4, SD, nullptr);
                else
                    dense_u12_col<float, W>(A + (size_t)k0 * ld + k0 + W + (it - n2), SL, ld);
            }
            __syncthreads();
            stamp(2 + 3 * (k0 / W), false);
            // ---- C: A22 -= L21 U12, 128 x 128 tiles on the tensor cores, column block by
            // column block (U12 staged once per block, L21 once per tile)
            const int tiles = (n2 + TC_M - 1) / TC_M;
            const int g = warp & 3, c = g * 32 + lane, rb = (warp >> 2) * 64;
            tc_stage_b(A, ld, k0, n2, 0, oper);
            tc_stage_a(A, ld, k0, n2, 0, oper);
            for (int t = 0; t < tiles * tiles; ++t) {
                const int tj = t / tiles, ti = t % tiles;
                const int row0 = ti * TC_M, col0 = tj * TC_N;
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncthreads();
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (tid == 0 && !wait_test) {
                    // the operand address through an opaque move, so that the 24 descriptors
                    // are formed here and not held in registers across the tile loop
                    uint32_t base;
                    asm volatile("mov.b32 %0, %1;" : "=r"(base) : "r"(smem_u32(oper)));
                    const uint32_t Ah = base, Al = base + TC_M * W * 4;
                    const uint32_t Bh = base + 2 * TC_M * W * 4, Bl = Bh + TC_N * W * 4;
                    // D^T = U12^T L21^T: the MMA's A operand is the U12 block (one row per tile
                    // column), its B operand the L21 rows, so that tensor-memory lane n holds
                    // column n of the update and a warp's tcgen05.ld covers 32 adjacent columns
                    const uint32_t As[3] = {Bh, Bl, Bh}, Bs[3] = {Ah, Ah, Al};
#pragma unroll
                    for (int pass = 0; pass < 3; ++pass) {
#pragma unroll
                        for (int j = 0; j < W / 8; ++j) {
                            const uint64_t da = tc_sdesc(As[pass] + 2 * j * LBO_B, LBO_B, 128);
                            const uint64_t db = tc_sdesc(Bs[pass] + 2 * j * LBO_A, LBO_A, 128);
                            const uint32_t accum = (pass | j) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(
                                    taddr),
                                "l"(da), "l"(db), "r"(idesc), "r"(accum));
                        }
                    }
                    asm volatile(
                        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                            smem_u32(&mbar))
                        : "memory");
                }
                // while the MMAs run: the next tile's rows of C go to L2, and this thread's first
                // 16 values of its tile column (column c, rows rb..rb + 63 of the tile: the
                // tensor-memory lane and column half its warp may read) are loaded
                if (t + 1 < tiles * tiles && tid < TC_M) {
                    const int nr0 = ((t + 1) % tiles) * TC_M, nc0 = ((t + 1) / tiles) * TC_N;
                    if (nr0 + tid < n2) {
                        const float* nrow = A + (size_t)(k0 + W + nr0 + tid) * ld + k0 + W + nc0;
#pragma unroll
                        for (int c = 0; c < TC_N; c += 32)
                            if (nc0 + c < n2) prefetch_l2(nrow + c);
                    }
                }
                // the thread's 64 values of C (one load of 32 adjacent columns per warp and row)
                // go in two halves of 32 rows, the first half's loads in flight while the MMAs
                // run; C - D is written back from tcgen05.ld registers, 16 rows at a time
                const bool cok = col0 + c < n2;
                float* cbase = A + (size_t)(k0 + W + row0 + rb) * ld + k0 + W + col0 + (cok ? c : 0);
                const int rows_left = cok ? n2 - row0 - rb : 0;  // rows of this half to update
                float cv[32];
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    if (j < rows_left) cv[j] = cbase[j * ld];
                const bool ok = tc_wait(smem_u32(&mbar), phase);
                if (__syncthreads_or(!ok)) {
                    // every thread agrees; the MMAs may still be running: wait once more
                    // (bounded) before the tensor memory is freed
                    tc_wait(smem_u32(&mbar), phase);
                    timed_out = 1;
                    break;
                }
                phase ^= 1u;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
                for (int half = 0; half < 2; ++half) {
                    float* ch = cbase + (size_t)(32 * half) * ld;
                    const int left = rows_left - 32 * half;
                    if (half == 1) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < left) cv[j] = ch[j * ld];
                    }
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        float d[16];
                        tc_ld16(taddr + ((uint32_t)(g * 32) << 16) + (uint32_t)(rb + 32 * half + 16 * h), d);
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            if (16 * h + j < left) ch[(16 * h + j) * ld] = cv[16 * h + j] - d[j];
                    }
                }
                // the next tile's operands (the MMAs have finished reading these buffers)
                if (t + 1 < tiles * tiles) {
                    const int tj1 = (t + 1) / tiles, ti1 = (t + 1) % tiles;
                    if (tj1 != tj) tc_stage_b(A, ld, k0, n2, tj1 * TC_N, oper);
                    tc_stage_a(A, ld, k0, n2, ti1 * TC_M, oper);
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            }
            // the panel's updates are visible to the next diagonal block
            __syncthreads();
            if (timed_out) break;
        } else {
            stamp(2 + 3 * (k0 / W), true);
        }
        stamp(3 + 3 * (k0 / W), false);
    }
    if (tid == 0 && (bad || timed_out)) B.singular[q] = 1;
    if (tid == 0 && timed_out) B.ctrl[5] = 1;
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(TC_N));
}

// The split path's trailing update on the tensor cores (FP32): one CTA per (128 x 128 tile of
// the trailing block, scenario) for the 32-column panel at k0 (its L21 and U12 written by
// k_dlu_panel), the tile computed as in k_dense_lu_tc -- operands staged hi / lo, 12 MMAs of the
// transposed product into tensor memory, C loaded while they run, C - D written back from
// tcgen05.ld registers.  Many CTAs per SM overlap one another's phases.  64 KB of operands, so
// at most three CTAs share an SM (3 x 128 tensor-memory columns); with k_dense_lu_tc's CTAs on
// the same SM, shared memory and registers still keep the columns in use below the SM's 512,
// so the allocation never waits.  The wait on the MMAs is bounded: when it runs out the
// scenario is marked singular and ctrl[5] set.
__global__ void __launch_bounds__(256, 3) k_dlu_update_tc(BatchDev B, int N, int k0, int tiles) {
    constexpr int W = TC_W;
    const int q = blockIdx.y;
    // a scenario already marked singular (a pivot, or a wait of an earlier panel that ran
    // out) is not updated further
    if (q >= B.n_scen || !B.solving[q] || B.singular[q] || (B.gfactor && !B.gfactor[q / B.sw]))
        return;
    const int ld = dense_ld(N);
    float* A = reinterpret_cast<float*>(B.Dt) + (size_t)q * N * ld;
    const bool wait_test = B.ctrl[6] != 0;  // test hook: issue no MMAs (the wait runs out)
    const int n2 = N - k0 - W;
    const int row0 = (blockIdx.x / tiles) * TC_M, col0 = (blockIdx.x % tiles) * TC_N;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* oper = smraw;
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tslot;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tslot)),
                     "r"(TC_N));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    tc_stage_b(A, ld, k0, n2, col0, oper);
    tc_stage_a(A, ld, k0, n2, row0, oper);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = tslot;
    if (tid == 0 && !wait_test) {
        // F32 accumulate, TF32 A and B, both K-major, N = 128, M = 128
        constexpr uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) |
                                   ((uint32_t)(TC_N >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
        constexpr uint32_t LBO_A = (TC_M / 8) * 128, LBO_B = (TC_N / 8) * 128;
        const uint32_t base = smem_u32(oper);
        const uint32_t Ah = base, Al = base + TC_M * W * 4;
        const uint32_t Bh = base + 2 * TC_M * W * 4, Bl = Bh + TC_N * W * 4;
        // D^T = U12^T L21^T: tensor-memory lane n holds column n of the update
        const uint32_t As[3] = {Bh, Bl, Bh}, Bs[3] = {Ah, Ah, Al};
#pragma unroll
        for (int pass = 0; pass < 3; ++pass) {
#pragma unroll
            for (int j = 0; j < W / 8; ++j) {
                const uint64_t da = tc_sdesc(As[pass] + 2 * j * LBO_B, LBO_B, 128);
                const uint64_t db = tc_sdesc(Bs[pass] + 2 * j * LBO_A, LBO_A, 128);
                const uint32_t accum = (pass | j) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(taddr),
                    "l"(da), "l"(db), "r"(idesc), "r"(accum));
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_u32(&mbar))
                     : "memory");
    }
    // this thread's tile column c and rows rb..rb + 63 (its warp's tensor-memory lane quarter
    // and column half), 16 rows at a time; the first 16 values of C load while the MMAs run
    const int g = warp & 3, c = g * 32 + lane, rb = (warp >> 2) * 64;
    const bool cok = col0 + c < n2;
    float* cbase = A + (size_t)(k0 + W + row0 + rb) * ld + k0 + W + col0 + (cok ? c : 0);
    const int rows_left = cok ? n2 - row0 - rb : 0;
    float cv[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (j < rows_left) cv[j] = cbase[j * ld];
    const bool ok = tc_wait(smem_u32(&mbar), 0u);
    if (__syncthreads_or(!ok)) {
        // every thread agrees; wait once more (bounded) for the MMAs before freeing the memory
        tc_wait(smem_u32(&mbar), 0u);
        if (tid == 0) {
            B.singular[q] = 1;
            B.ctrl[5] = 1;
        }
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll 1
        for (int h = 0; h < 4; ++h) {
            float* ch = cbase + (size_t)(16 * h) * ld;
            const int left = rows_left - 16 * h;
            if (h > 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (j < left) cv[j] = ch[j * ld];
            }
            float d[16];
            tc_ld16(taddr + ((uint32_t)(g * 32) << 16) + (uint32_t)(rb + 16 * h), d);
#pragma unroll
            for (int j = 0; j < 16; ++j)
                if (j < left) ch[j * ld] = cv[j] - d[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(TC_N));
}

// Dynamic shared memory of k_dense_lu_tc.
__host__ __device__ __forceinline__ size_t dense_lu_tc_smem() {
    return (size_t)TC_OPER_BYTES + (2 * TC_W * (TC_W + 4) + TC_W) * 4;
}

}  // namespace gapk
