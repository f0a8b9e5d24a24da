// pt_mlp.cu — the radiance-cache MLP on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Network: 64 inputs (position frequency encoding 3x12, spherical harmonics of the direction up
// to degree 3 = 16 coefficients, normal, albedo, roughness = 7; zero padded), five hidden layers
// of 64 with ReLU, 3 outputs with exp.  BF16 weights and activations, FP32 accumulation in TMEM.
// No counterpart in the reference (it has no learned component).
//
// Shared-memory operand layout (one convention for every matrix): a R x C bf16 matrix is stored
// as 8-row x 8-column core matrices of 128 contiguous bytes; element (r, c) sits at byte
//   (r % 8) * 16 + (r / 8) * (C / 8) * 128 + (c % 8) * 2 + (c / 8) * 128.
// Read with rows as M/N and columns as K it is the canonical K-major no-swizzle layout
// (LBO = 128 B between K core matrices, SBO = C*16 B between row groups); read transposed it is
// the canonical MN-major layout (SBO = 128 B, LBO = C*16 B).  So activations, gradients and
// weights are each stored once and used both ways: X*W, dZ*W^T and X^T*dZ.
// Every mbarrier wait is bounded: on expiry the kernel records PT_TIMEOUT in its status word and
// stops issuing; a group whose wait ran out then waits once more, with the full limit, for the
// MMAs it had committed (so no MMA still writes TMEM), frees its TMEM and returns.  The reduce and
// Adam kernels leave the weights alone while the status word is set.
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_bf16.h>
#include "pt_api_common.h"
#include "pt_device.h"

using namespace ptb;

namespace ptb {
namespace mlp {

constexpr int kTile = 128;             // rows per MMA tile (queries)
constexpr int kWidth = 64;             // input and hidden width
constexpr int kHidden = 5;             // hidden layers (matrices 0..4 are 64x64)
constexpr int kOut = 3;
constexpr int kOutPad = 16;            // output layer N, padded for M = 128
constexpr int kMatBytes = kWidth * kWidth * 2;             // 8 KB
constexpr int kOutMatBytes = kOutPad * kWidth * 2;         // 2 KB
constexpr int kWeightBytes = kHidden * kMatBytes + kOutMatBytes;   // 43008
constexpr int kActBytes = kTile * kWidth * 2;              // 16 KB per 128 x 64 tile
constexpr int kOutActBytes = kTile * kOutPad * 2;          // 4 KB per 128 x 16 tile
constexpr int kPad = 2048;                                 // guard after every operand buffer
constexpr int kMasterFloats = kHidden * kWidth * kWidth + kWidth * kOut;   // 20672
constexpr long long kSpinLimit = 1ll << 22;   // mbarrier try_wait attempts before a wait gives up

// byte offset of element (r, c) of a matrix with `cols` columns in the core-matrix layout
__host__ __device__ inline uint32_t canon(uint32_t r, uint32_t c, uint32_t cols) {
    return (r % 8) * 16 + (r / 8) * (cols / 8) * 128 + (c % 8) * 2 + (c / 8) * 128;
}

__device__ inline uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// UMMA shared-memory descriptor, no swizzle, Blackwell version bit
__device__ inline uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// instruction descriptor: kind::f16, BF16 x BF16 -> F32
__host__ __device__ constexpr uint32_t idesc(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ inline void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                 :: "r"(d_tmem), "l"(a), "l"(b), "r"(id), "r"(accumulate));
}
__device__ inline void commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ inline void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ inline void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ inline void wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ inline void bar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// bounded wait for the phase with parity `phase` to complete: at most `attempts` try_waits
__device__ inline bool bar_wait(uint64_t *bar, uint32_t phase, long long attempts) {
    uint32_t addr = smem_u32(bar);
    for (long long i = 0; i < attempts; i++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n" : "=r"(done) : "r"(addr), "r"(phase) : "memory");
        if (done) return true;
    }
    return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31)
__device__ inline void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    wait_ld();
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// writes 8 bf16 values (columns 8c..8c+7 of row r) into a core-matrix layout buffer
__device__ inline void store8(unsigned char *base, uint32_t r, uint32_t c8, uint32_t cols, const float *x) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(x[0], x[1]), p1 = __floats2bfloat162_rn(x[2], x[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(x[4], x[5]), p3 = __floats2bfloat162_rn(x[6], x[7]);
    uint4 v;
    v.x = *reinterpret_cast<uint32_t *>(&p0); v.y = *reinterpret_cast<uint32_t *>(&p1);
    v.z = *reinterpret_cast<uint32_t *>(&p2); v.w = *reinterpret_cast<uint32_t *>(&p3);
    *reinterpret_cast<uint4 *>(base + canon(r, c8 * 8, cols)) = v;
}
// store8 of max(x, 0): the conversion instruction applies the ReLU
__device__ inline void store8_relu(unsigned char *base, uint32_t r, uint32_t c8, uint32_t cols, const float *x) {
    uint4 v;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(v.x) : "f"(x[1]), "f"(x[0]));
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(v.y) : "f"(x[3]), "f"(x[2]));
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(v.z) : "f"(x[5]), "f"(x[4]));
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(v.w) : "f"(x[7]), "f"(x[6]));
    *reinterpret_cast<uint4 *>(base + canon(r, c8 * 8, cols)) = v;
}
__device__ inline void load8(const unsigned char *base, uint32_t r, uint32_t c8, uint32_t cols, float *x) {
    uint4 v = *reinterpret_cast<const uint4 *>(base + canon(r, c8 * 8, cols));
    const __nv_bfloat162 *p = reinterpret_cast<const __nv_bfloat162 *>(&v);
#pragma unroll
    for (int i = 0; i < 4; i++) { float2 f = __bfloat1622float2(p[i]); x[2 * i] = f.x; x[2 * i + 1] = f.y; }
}

// Collects a row's encoded values eight at a time and stores each group of eight as soon as it is
// complete, so a thread holds at most eight of its 64 inputs in registers.
struct RowWriter {
    unsigned char *base;
    uint32_t r;
    float buf[8];
    int k = 0;
    __device__ __forceinline__ void operator()(float v) {
        buf[k & 7] = v;
        if ((++k & 7) == 0) store8(base, r, uint32_t(k / 8 - 1), 64, buf);
    }
};

// Input encoding of one query (see the file comment); 64 values, zero padded.
__device__ __forceinline__ void encode(const pt_cache_query &q, float3 lo, float3 inv_extent, RowWriter &put) {
    const float p3[3] = {(q.position.x - lo.x) * inv_extent.x, (q.position.y - lo.y) * inv_extent.y,
                         (q.position.z - lo.z) * inv_extent.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        float sn, cs;
        sincosf(3.14159265358979f * p3[a], &sn, &cs);
#pragma unroll
        for (int f = 0; f < 6; f++) {          // frequencies 2^f pi p by the double-angle identities
            put(sn); put(cs);
            float s2 = 2.0f * sn * cs;
            cs = (cs - sn) * (cs + sn);
            sn = s2;
        }
    }
    float dx = q.direction.x, dy = q.direction.y, dz = q.direction.z;
    float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    put(0.28209479177387814f);
    put(-0.48860251190291987f * dy);
    put(0.48860251190291987f * dz);
    put(-0.48860251190291987f * dx);
    put(1.0925484305920792f * dx * dy);
    put(-1.0925484305920792f * dy * dz);
    put(0.31539156525252005f * (3.0f * zz - 1.0f));
    put(-1.0925484305920792f * dx * dz);
    put(0.5462742152960396f * (xx - yy));
    put(-0.5900435899266435f * dy * (3.0f * xx - yy));
    put(2.890611442640554f * dx * dy * dz);
    put(-0.4570457994644658f * dy * (5.0f * zz - 1.0f));
    put(0.3731763325901154f * dz * (5.0f * zz - 3.0f));
    put(-0.4570457994644658f * dx * (5.0f * zz - 1.0f));
    put(1.445305721320277f * dz * (xx - yy));
    put(-0.5900435899266435f * dx * (xx - 3.0f * yy));
    put(q.normal.x); put(q.normal.y); put(q.normal.z);
    put(q.albedo.x); put(q.albedo.y); put(q.albedo.z);
    put(q.roughness);
#pragma unroll
    for (int i = 0; i < 5; i++) put(0.0f);
}

struct Scratch {                // per-CTA shared memory header
    uint64_t bar;
    uint32_t tmem;
    uint32_t pad[13];
};

__device__ inline void tmem_alloc(Scratch *h, uint32_t cols) {
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(&h->tmem)), "r"(cols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
}
__device__ inline void tmem_free(uint32_t base, uint32_t cols) {
    if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(base), "r"(cols) : "memory");
}

// Copies the canonical BF16 weights (global) into shared memory.
__device__ inline void load_weights(unsigned char *w, const unsigned char *g) {
    for (int i = threadIdx.x; i < kWeightBytes / 16; i += blockDim.x)
        reinterpret_cast<uint4 *>(w)[i] = reinterpret_cast<const uint4 *>(g)[i];
}

// X (128 x 64, rows = queries) into the core-matrix layout; rows past `count` are zero.
// `r` is the calling thread's row of the tile.
__device__ inline void encode_tile(unsigned char *x, const pt_cache_query *q, size_t first, size_t count, float3 lo,
                                   float3 inv_extent, uint32_t r) {
    size_t row = first + r;
    if (row < count) {
        RowWriter put{x, r};
        encode(q[row], lo, inv_extent, put);
    } else {
        const float zero[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int c = 0; c < 8; c++) store8(x, r, c, 64, zero);
    }
}

// D[128 x N] (+)= A[128 x K] * B[N x K]^T, A and B K-major in the core layout, K = 16 per MMA.
__device__ inline void mma_kk(uint32_t d, const unsigned char *a, uint32_t a_cols, const unsigned char *b, uint32_t b_cols,
                              int N, int K, bool accumulate) {
    for (int s = 0; s < K / 16; s++) {
        uint64_t da = desc(smem_u32(a) + s * 256, 128, a_cols * 16);
        uint64_t db = desc(smem_u32(b) + s * 256, 128, b_cols * 16);
        mma(d, da, db, idesc(kTile, N, false, false), (accumulate || s) ? 1u : 0u);
    }
}
// D[128 x N] (+)= A[128 x K] * B where B is stored as [K rows x N cols] (core layout): B read
// MN-major.  A K-major with a_cols = K.
__device__ inline void mma_kmn(uint32_t d, const unsigned char *a, uint32_t a_cols, const unsigned char *b, uint32_t b_cols,
                               int N, int K, bool accumulate) {
    for (int s = 0; s < K / 16; s++) {
        uint64_t da = desc(smem_u32(a) + s * 256, 128, a_cols * 16);
        uint64_t db = desc(smem_u32(b) + s * 2 * b_cols * 16, b_cols * 16, 128);
        mma(d, da, db, idesc(kTile, N, false, true), (accumulate || s) ? 1u : 0u);
    }
}
// D[128(64 valid) x N] (+)= A^T * B with A [128 rows m x 64 cols k] and B [128 rows m x N cols],
// both read MN-major (the reduction runs over the 128 rows m).
__device__ inline void mma_tn(uint32_t d, const unsigned char *a, const unsigned char *b, uint32_t b_cols, int N, bool accumulate) {
    for (int s = 0; s < kTile / 16; s++) {
        uint64_t da = desc(smem_u32(a) + s * 2 * 64 * 16, 64 * 16, 128);
        uint64_t db = desc(smem_u32(b) + s * 2 * b_cols * 16, b_cols * 16, 128);
        mma(d, da, db, idesc(kTile, N, true, true), (accumulate || s) ? 1u : 0u);
    }
}

// Thread 0 commits the MMAs it issued to the barrier; every thread waits (bounded).  Returns, the
// same in every thread of the CTA, whether all of them saw the MMAs complete.
struct Sync {
    Scratch *h;
    long long attempts;
    uint32_t phase = 0;
    bool pending = false;       // this thread's wait ran out on phase pending_phase
    uint32_t pending_phase = 0;
    __device__ bool wait_all() {
        if (threadIdx.x == 0) commit(&h->bar);
        bool ok = bar_wait(&h->bar, phase, attempts);
        if (!ok) { pending = true; pending_phase = phase; }
        phase ^= 1;
        ok = __syncthreads_and(ok) != 0;
        fence_after();
        return ok;
    }
    // after a wait that ran out: wait, with the full limit, for the committed MMAs to finish
    __device__ void drain() {
        if (pending) bar_wait(&h->bar, pending_phase, kSpinLimit);
    }
};

// ---- forward (query) -----------------------------------------------------------------------
// A CTA runs kFwdGroups independent tile pipelines ("groups" of four warps, one 128-query tile
// each) over one shared copy of the weights.  Group g owns TMEM columns [64g, 64g + 64) (each
// hidden layer's 128 x 64 accumulator, then the 128 x 16 output in the same columns), one
// activation buffer, one mbarrier and named barrier 1 + g.  One activation buffer suffices: each
// layer's epilogue runs after that layer's MMA has completed, so it overwrites the MMA's own input.
// smem: header (Scratch, then the groups' mbarriers from byte 128) | W | pad | (act | pad) x G.
// One CTA of eight groups per SM: eight tiles in flight (32 warps at 64 registers), all 512
// TMEM columns, 188 KB of shared memory.
constexpr int kFwdGroups = 8;
constexpr int kFwdThreads = kFwdGroups * kTile;
constexpr int kFwdCtasPerSm = 1;
constexpr uint32_t kFwdTmemCols = 512;    // power of two >= 64 * kFwdGroups
constexpr size_t kFwdSmem = 256 + kWeightBytes + kPad + kFwdGroups * (kActBytes + kPad);
static_assert(64 * kFwdGroups <= kFwdTmemCols && kFwdCtasPerSm * kFwdTmemCols <= 512, "TMEM budget");
static_assert(128 + 8 * kFwdGroups <= 256 && kFwdGroups < 16, "header and named-barrier budget");

// named barrier over one group's 128 threads; returns whether every thread passed `ok`
__device__ inline bool group_sync_and(int id, bool ok) {
    uint32_t r;
    asm volatile("{\n\t.reg .pred p, q;\n\tsetp.ne.b32 p, %1, 0;\n\t"
                 "barrier.cta.red.and.pred q, %2, 128, p;\n\tselp.b32 %0, 1, 0, q;\n\t}\n"
                 : "=r"(r) : "r"((uint32_t)ok), "r"(id) : "memory");
    return r != 0;
}

__global__ void __launch_bounds__(kFwdThreads, kFwdCtasPerSm) forward_kernel(const unsigned char *weights,
                                                                             const pt_cache_query *queries, size_t count,
                                                                             const int32_t *count_dev, float3 lo, float3 hi,
                                                                             float *out, int *status, long long attempts) {
    if (count_dev) count = min(count, size_t(max(0, *count_dev)));   // queue length known only on the device
    extern __shared__ __align__(1024) unsigned char smem[];
    Scratch *h = reinterpret_cast<Scratch *>(smem);
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 128);
    unsigned char *w = smem + 256;
    const int g = threadIdx.x / kTile;
    const uint32_t r = threadIdx.x % kTile;                        // this thread's row of its group's tile
    unsigned char *act = w + kWeightBytes + kPad + size_t(g) * (kActBytes + kPad);
    const float3 ie = make_float3(1.0f / fmaxf(hi.x - lo.x, 1e-30f), 1.0f / fmaxf(hi.y - lo.y, 1e-30f), 1.0f / fmaxf(hi.z - lo.z, 1e-30f));
    if (threadIdx.x < kFwdGroups) bar_init(&bars[threadIdx.x]);
    tmem_alloc(h, kFwdTmemCols);
    load_weights(w, weights);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tcol = h->tmem + 64u * uint32_t(g);
    const uint32_t lane_col = tcol + ((uint32_t)((r & ~31u)) << 16);   // warp (w % 4) reads lanes 32 (w % 4) ..
    uint64_t *bar = &bars[g];
    const bool issuer = r == 0;
    uint32_t phase = 0, pending_phase = 0;
    bool ok = true, pending = false;
    auto wait_mma = [&]() {                       // commit this group's MMAs and wait for them (bounded)
        if (issuer) commit(bar);
        bool done = bar_wait(bar, phase, attempts);
        if (!done) { pending = true; pending_phase = phase; }
        phase ^= 1;
        fence_after();
        return done;
    };
    auto sync_group = [&](bool v) {
        fence_async_smem();
        fence_before();
        bool all = group_sync_and(1 + g, v);
        fence_after();
        return all;
    };
    const uint32_t tiles = uint32_t((count + kTile - 1) / kTile);   // < 2^32: 2^39 queries would not fit in memory
    const uint32_t stride = gridDim.x * kFwdGroups;
    for (uint32_t t = blockIdx.x * kFwdGroups + g; t < tiles && ok; t += stride) {
        encode_tile(act, queries, size_t(t) * kTile, count, lo, ie, r);
        sync_group(true);
        for (int layer = 0; layer < kHidden && ok; layer++) {
            if (issuer) mma_kk(tcol, act, 64, w + layer * kMatBytes, 64, 64, 64, false);
            bool done = wait_mma();               // the MMA has read all of act: its rows may be overwritten
            if (done) {
                for (int c = 0; c < 4; c++) {
                    float v[16];
                    tmem_ld16(lane_col + c * 16, v);
                    store8_relu(act, r, 2 * c, 64, v);
                    store8_relu(act, r, 2 * c + 1, 64, v + 8);
                }
            }
            ok = sync_group(done);
        }
        if (!ok) break;
        if (issuer) mma_kk(tcol, act, 64, w + kHidden * kMatBytes, 64, kOutPad, 64, false);
        bool done = wait_mma();
        if (done) {
            float v[16];
            tmem_ld16(lane_col, v);
            size_t row = size_t(t) * kTile + r;
            if (row < count) { out[3 * row] = expf(v[0]); out[3 * row + 1] = expf(v[1]); out[3 * row + 2] = expf(v[2]); }
        }
        ok = sync_group(done);                    // the next tile's MMAs write these TMEM columns again
    }
    if (!ok && r == 0) atomicExch(status, int(PT_TIMEOUT));
    if (pending) bar_wait(bar, pending_phase, kSpinLimit);   // no MMA of this group may still write TMEM
    fence_before();
    __syncthreads();
    tmem_free(h->tmem, kFwdTmemCols);
}

// ---- training (forward + relative-L2 loss + backward) --------------------------------------
// TMEM columns: [0,64) forward scratch, [64,80) output, [96,112) dW5, [128,192) dH scratch,
// [192 + 64 l, 256 + 64 l) dW_l for l = 0..4.
// smem: header | W | pad | H0..H5 (each + pad) | dZ + pad | dZ5 + pad
constexpr size_t kTrainSmem = 256 + kWeightBytes + kPad + 6 * (kActBytes + kPad) + (kActBytes + kPad) + (kOutActBytes + kPad);

__global__ void __launch_bounds__(kTile, 1) train_kernel(const unsigned char *weights, const pt_cache_query *queries,
                                                         const float *targets, size_t count, const int32_t *count_dev,
                                                         float3 lo, float3 hi, float *partial, float *loss_partial, int *status,
                                                         long long attempts) {
    if (count_dev) count = min(count, size_t(max(0, *count_dev)));
    const float grad_scale = count ? 1.0f / float(count * kOut) : 0.0f;   // mean over samples and channels
    extern __shared__ __align__(1024) unsigned char smem[];
    Scratch *h = reinterpret_cast<Scratch *>(smem);
    unsigned char *w = smem + 256;
    unsigned char *act[6];
    act[0] = w + kWeightBytes + kPad;
    for (int i = 1; i < 6; i++) act[i] = act[i - 1] + kActBytes + kPad;
    unsigned char *dz = act[5] + kActBytes + kPad;
    unsigned char *dz5 = dz + kActBytes + kPad;
    const float3 ie = make_float3(1.0f / fmaxf(hi.x - lo.x, 1e-30f), 1.0f / fmaxf(hi.y - lo.y, 1e-30f), 1.0f / fmaxf(hi.z - lo.z, 1e-30f));
    if (threadIdx.x == 0) bar_init(&h->bar);
    tmem_alloc(h, 512);
    load_weights(w, weights);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tbase = h->tmem;
    const uint32_t lane_base = tbase + ((uint32_t)(threadIdx.x & ~31u) << 16);
    Sync sync{h, attempts};
    bool ok = true, first = true;
    float loss = 0.0f;
    const size_t tiles = (count + kTile - 1) / kTile;
    for (size_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const size_t row = t * kTile + threadIdx.x;
        encode_tile(act[0], queries, t * kTile, count, lo, ie, threadIdx.x);
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        for (int layer = 0; layer < kHidden && ok; layer++) {
            if (threadIdx.x == 0) mma_kk(tbase, act[layer], 64, w + layer * kMatBytes, 64, 64, 64, false);
            ok = sync.wait_all();
            if (!ok) break;
            for (int c = 0; c < 4; c++) {
                float v[16];
                tmem_ld16(lane_base + c * 16, v);
                store8_relu(act[layer + 1], threadIdx.x, 2 * c, 64, v);
                store8_relu(act[layer + 1], threadIdx.x, 2 * c + 1, 64, v + 8);
            }
            fence_async_smem();
            fence_before();
            __syncthreads();
            fence_after();
        }
        if (!ok) break;
        if (threadIdx.x == 0) mma_kk(tbase + 64, act[5], 64, w + kHidden * kMatBytes, 64, kOutPad, 64, false);
        ok = sync.wait_all();
        if (!ok) break;
        {
            // relative L2 loss, sum_c (y - t)^2 / (sg(y)^2 + 0.01) with y = exp(z): dL/dz = 2 (y - t) y / (y^2 + 0.01)
            float v[16], g[16];
            tmem_ld16(lane_base + 64, v);
            for (int i = 0; i < 16; i++) g[i] = 0.0f;
            if (row < count) {
                for (int c = 0; c < kOut; c++) {
                    float y = expf(v[c]), target = targets[3 * row + c];
                    float denom = y * y + 0.01f, diff = y - target;
                    loss += diff * diff / denom;
                    g[c] = grad_scale * 2.0f * diff * y / denom;
                }
            }
            store8(dz5, threadIdx.x, 0, kOutPad, g);
            store8(dz5, threadIdx.x, 1, kOutPad, g + 8);
        }
        fence_async_smem();
        fence_before();
        __syncthreads();
        fence_after();
        // dW5 += H5^T dZ5 ; dH5 = dZ5 W5^T
        if (threadIdx.x == 0) {
            mma_tn(tbase + 96, act[5], dz5, kOutPad, kOutPad, !first);
            mma_kmn(tbase + 128, dz5, kOutPad, w + kHidden * kMatBytes, 64, 64, kOutPad, false);
        }
        ok = sync.wait_all();
        if (!ok) break;
        for (int layer = kHidden - 1; layer >= 0 && ok; layer--) {
            // dZ_layer = dH_{layer+1} * [H_{layer+1} > 0]
            for (int c = 0; c < 4; c++) {
                float v[16], a[16];
                tmem_ld16(lane_base + 128 + c * 16, v);
                load8(act[layer + 1], threadIdx.x, 2 * c, 64, a);
                load8(act[layer + 1], threadIdx.x, 2 * c + 1, 64, a + 8);
                for (int i = 0; i < 16; i++) v[i] = a[i] > 0.0f ? v[i] : 0.0f;
                store8(dz, threadIdx.x, 2 * c, 64, v);
                store8(dz, threadIdx.x, 2 * c + 1, 64, v + 8);
            }
            fence_async_smem();
            fence_before();
            __syncthreads();
            fence_after();
            if (threadIdx.x == 0) {
                mma_tn(tbase + 192 + 64 * layer, act[layer], dz, 64, 64, !first);        // dW_layer += H^T dZ
                if (layer > 0) mma_kmn(tbase + 128, dz, 64, w + layer * kMatBytes, 64, 64, 64, false);   // dH = dZ W^T
            }
            ok = sync.wait_all();
        }
        first = false;
    }
    // per-CTA partial gradients (rows k of the dW accumulators live in TMEM lanes 0..63)
    float *mine = partial + size_t(blockIdx.x) * kMasterFloats;
    if (ok) {
        for (int layer = 0; layer < kHidden; layer++) {
            for (int c = 0; c < 4; c++) {
                float v[16];
                tmem_ld16(lane_base + 192 + 64 * layer + c * 16, v);
                if (threadIdx.x < 64)
                    for (int i = 0; i < 16; i++) mine[layer * 4096 + threadIdx.x * 64 + c * 16 + i] = first ? 0.0f : v[i];
            }
        }
        float v[16];
        tmem_ld16(lane_base + 96, v);
        if (threadIdx.x < 64)
            for (int i = 0; i < kOut; i++) mine[kHidden * 4096 + threadIdx.x * kOut + i] = first ? 0.0f : v[i];
    }
    // loss partial
    for (int o = 16; o; o >>= 1) loss += __shfl_down_sync(0xffffffffu, loss, o);
    __shared__ float warp_loss[4];
    if ((threadIdx.x & 31) == 0) warp_loss[threadIdx.x >> 5] = loss;
    __syncthreads();
    if (threadIdx.x == 0) loss_partial[blockIdx.x] = warp_loss[0] + warp_loss[1] + warp_loss[2] + warp_loss[3];
    if (!ok && threadIdx.x == 0) atomicExch(status, int(PT_TIMEOUT));
    sync.drain();                                 // no MMA may still write TMEM when it is freed
    fence_before();
    __syncthreads();
    tmem_free(tbase, 512);
}

// FP32 master weight i -> its bf16 position in the canonical buffer.
__host__ __device__ inline uint32_t master_to_canon(int i) {
    if (i < kHidden * 4096) {
        int layer = i / 4096, k = (i % 4096) / 64, n = i % 64;          // master W[k][n], stored as Wt rows n cols k
        return uint32_t(layer * kMatBytes) + canon(uint32_t(n), uint32_t(k), 64);
    }
    int j = i - kHidden * 4096, k = j / kOut, n = j % kOut;
    return uint32_t(kHidden * kMatBytes) + canon(uint32_t(n), uint32_t(k), 64);
}

struct AdamArgs {
    float *master, *m, *v;
    float lr, beta1, beta2, eps;
    unsigned char *canon_out;           // bf16 canonical copy of the masters
    float ema_decay;                    // > 0: also keep the weight average and its bf16 copy
    float *ema;
    unsigned char *ema_canon;
};

constexpr int kReduceSlices = 8;        // warps per block; warp k sums the partials of CTAs k, k + 8, ...

// Sums the per-CTA partial gradients into `grad` and, with kAdam on a non-empty batch, applies
// one bias-corrected Adam step to the FP32 masters and writes their bf16 canonical copy (and the
// weight average with its copy).  One block of 8 warps per 32 masters: warp k sums the rows of
// CTAs k, k + 8, ... (each row read as one 128-byte line), then warp 0 adds the eight sums in a
// fixed order, so the result is deterministic.  Every block reads the step counters as they were
// before this step and uses step + 1; the last block to finish (completion counter `done`, reset
// by that block) writes the mean loss into loss[0] and, with `advance` on a non-empty batch,
// advances the Adam step (step[0]) and the weight-average step (step[1]).  Nothing happens when
// the gradient kernel timed out (*status).
template <bool kAdam>
__global__ void __launch_bounds__(32 * kReduceSlices) reduce_step_kernel(const float *partial, const float *loss_partial, int ctas,
                                                                         size_t count, const int32_t *count_dev, float *grad,
                                                                         float *loss, int *step, unsigned *done, int advance,
                                                                         AdamArgs a, const int *status) {
    if (*status) return;
    __shared__ float sums[kReduceSlices][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, slice = threadIdx.x >> 5;
    const int i = blockIdx.x * 32 + lane;
    const size_t n = count_dev ? min(count, size_t(max(0, *count_dev))) : count;
    float s = 0.0f;
    if (i < kMasterFloats)
        for (int c = slice; c < ctas; c += kReduceSlices) s += partial[size_t(c) * kMasterFloats + i];
    sums[slice][lane] = s;
    __syncthreads();
    if (slice == 0 && i < kMasterFloats) {
        float g = sums[0][lane];
#pragma unroll
        for (int k = 1; k < kReduceSlices; k++) g += sums[k][lane];
        grad[i] = g;
        if (kAdam && n) {
            const int t = step[0] + 1;
            float mi = a.beta1 * a.m[i] + (1.0f - a.beta1) * g;
            float vi = a.beta2 * a.v[i] + (1.0f - a.beta2) * g * g;
            a.m[i] = mi; a.v[i] = vi;
            float mh = mi / (1.0f - powf(a.beta1, float(t))), vh = vi / (1.0f - powf(a.beta2, float(t)));
            float w = a.master[i] - a.lr * mh / (sqrtf(vh) + a.eps);
            a.master[i] = w;
            const uint32_t at = master_to_canon(i);
            *reinterpret_cast<__nv_bfloat16 *>(a.canon_out + at) = __float2bfloat16_rn(w);
            if (a.ema_decay > 0.0f) {
                float e = a.ema_decay * a.ema[i] + (1.0f - a.ema_decay) * w;
                a.ema[i] = e;
                float corrected = e / (1.0f - powf(a.ema_decay, float(step[1] + 1)));
                *reinterpret_cast<__nv_bfloat16 *>(a.ema_canon + at) = __float2bfloat16_rn(corrected);
            }
        }
    }
    __syncthreads();                    // this block's reads of step[] are done
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        float l = 0.0f;
        for (int c = 0; c < ctas; c++) l += loss_partial[c];
        loss[0] = n ? l / float(n * kOut) : 0.0f;
        if (n && advance) { step[0] += 1; step[1] += 1; }
        *done = 0;
    }
}

__global__ void canon_kernel(const float *master, unsigned char *canon_out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kMasterFloats) return;
    *reinterpret_cast<__nv_bfloat16 *>(canon_out + master_to_canon(i)) = __float2bfloat16_rn(master[i]);
}

} // namespace mlp
} // namespace ptb

using namespace ptb::mlp;

struct pt_cache {
    DeviceBuffer master, adam_m, adam_v, grad, weights, partial, loss_partial, status, step, loss;
    DeviceBuffer done;                  // completion counter of the reduction (zero between launches)
    DeviceBuffer ema, ema_weights;      // weight average and its bf16 copy (used for inference when ema_decay > 0)
    float lo[3], hi[3];
    int ctas = 0;
    float lr = 1e-2f, beta1 = 0.9f, beta2 = 0.99f, eps = 1e-8f;
    float ema_decay = 0.0f;
    long long attempts = kSpinLimit;    // try_wait attempts per bounded wait (pt_cache_wait_limit)
    const unsigned char *inference() const { return (ema_decay > 0 ? ema_weights : weights).get<unsigned char>(); }
};

namespace {
// bf16 copies from the masters; the weight average restarts from them (step[1] = 0)
void refresh_canon(pt_cache *c, cudaStream_t st) {
    canon_kernel<<<(kMasterFloats + 255) / 256, 256, 0, st>>>(c->master.get<float>(), c->weights.get<unsigned char>());
    PT_CUDA(cudaGetLastError());
    PT_CUDA(cudaMemcpyAsync(c->ema_weights.get(), c->weights.get(), kWeightBytes, cudaMemcpyDeviceToDevice, st));
    PT_CUDA(cudaMemsetAsync(c->ema.get(), 0, kMasterFloats * sizeof(float), st));
    PT_CUDA(cudaMemsetAsync(c->step.get<int>() + 1, 0, sizeof(int), st));
}
void check_status(pt_cache *c) {
    int status = 0;
    PT_CUDA(cudaMemcpy(&status, c->status.get(), sizeof status, cudaMemcpyDeviceToHost));
    if (status) {
        PT_CUDA(cudaMemset(c->status.get(), 0, sizeof(int)));
        throw Error(pt_status(status), "radiance-cache kernel timed out waiting for the tensor cores");
    }
}
float3 lo3(const pt_cache *c) { return make_float3(c->lo[0], c->lo[1], c->lo[2]); }
float3 hi3(const pt_cache *c) { return make_float3(c->hi[0], c->hi[1], c->hi[2]); }
// forward/backward/reduce into c->grad and c->loss and, for a training step, the Adam update in
// the same reduction launch; no host synchronisation
void gradients(pt_cache *c, const pt_cache_query *q, const float *targets, size_t count, const int32_t *count_dev, bool train,
               cudaStream_t st) {
    size_t tiles = (count + kTile - 1) / kTile;
    int grid = count_dev ? c->ctas : int(std::min<size_t>(tiles ? tiles : 1, size_t(c->ctas)));
    train_kernel<<<grid, kTile, kTrainSmem, st>>>(c->weights.get<unsigned char>(), q, targets, count, count_dev, lo3(c), hi3(c),
                                                   c->partial.get<float>(), c->loss_partial.get<float>(), c->status.get<int>(),
                                                   c->attempts);
    PT_CUDA(cudaGetLastError());
    AdamArgs a{c->master.get<float>(), c->adam_m.get<float>(), c->adam_v.get<float>(), c->lr, c->beta1, c->beta2, c->eps,
               c->weights.get<unsigned char>(), c->ema_decay, c->ema.get<float>(), c->ema_weights.get<unsigned char>()};
    const unsigned blocks = unsigned((kMasterFloats + 31) / 32);
    auto kernel = train ? reduce_step_kernel<true> : reduce_step_kernel<false>;
    kernel<<<blocks, 32 * kReduceSlices, 0, st>>>(c->partial.get<float>(), c->loss_partial.get<float>(), grid, count, count_dev,
                                                   c->grad.get<float>(), c->loss.get<float>(), c->step.get<int>(),
                                                   c->done.get<unsigned>(), train ? 1 : 0, a, c->status.get<int>());
    PT_CUDA(cudaGetLastError());
}
float read_loss(pt_cache *c, cudaStream_t st) {
    float l = 0;
    PT_CUDA(cudaMemcpyAsync(&l, c->loss.get(), sizeof l, cudaMemcpyDeviceToHost, st));
    PT_CUDA(cudaStreamSynchronize(st));
    check_status(c);
    return l;
}
} // namespace

namespace ptb {
void cache_bounds(const pt_cache *c, float lo[3], float hi[3]) {
    for (int a = 0; a < 3; a++) { lo[a] = c->lo[a]; hi[a] = c->hi[a]; }
}
void cache_forward(pt_cache *c, const pt_cache_query *queries, size_t count, const int32_t *count_dev, float *rgb, cudaStream_t st) {
    size_t tiles = (count + kTile - 1) / kTile;
    if (!tiles) return;
    int grid = int(std::min<size_t>((tiles + kFwdGroups - 1) / kFwdGroups, size_t(kFwdCtasPerSm) * size_t(c->ctas)));
    forward_kernel<<<grid, kFwdThreads, kFwdSmem, st>>>(c->inference(), queries, count, count_dev, lo3(c), hi3(c), rgb,
                                                   c->status.get<int>(), c->attempts);
    PT_CUDA(cudaGetLastError());
}
void cache_train(pt_cache *c, const pt_cache_query *queries, const float *targets, size_t count, const int32_t *count_dev,
                 cudaStream_t st) {
    if (!count) return;
    gradients(c, queries, targets, count, count_dev, true, st);
}
float cache_loss(pt_cache *c, cudaStream_t st) { return read_loss(c, st); }
void cache_status(pt_cache *c) { check_status(c); }
} // namespace ptb

extern "C" {

pt_status pt_cache_create(const float scene_lo[3], const float scene_hi[3], uint64_t seed, pt_cache **out) {
    return guard([&]() {
        if (!scene_lo || !scene_hi || !out) throw Error(PT_INVALID_ARGUMENT, "null argument");
        *out = nullptr;
        require_device();
        auto c = new pt_cache;
        try {
            for (int a = 0; a < 3; a++) { c->lo[a] = scene_lo[a]; c->hi[a] = scene_hi[a]; }
            // Uniform(-sqrt(6/(fan_in+fan_out)), +) initialisation from a splitmix64 stream
            std::vector<float> w(kMasterFloats);
            uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
            auto uniform = [&]() {
                uint64_t z = (s += 0x9E3779B97F4A7C15ull);
                z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
                z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
                z ^= z >> 31;
                return double(z >> 11) * 0x1p-53;
            };
            for (int i = 0; i < kMasterFloats; i++) {
                double bound = i < kHidden * 4096 ? std::sqrt(6.0 / 128.0) : std::sqrt(6.0 / 67.0);
                w[size_t(i)] = float((2 * uniform() - 1) * bound);
            }
            c->master.upload(w);
            std::vector<float> zeros(kMasterFloats, 0.0f);
            c->adam_m.upload(zeros); c->adam_v.upload(zeros); c->grad.upload(zeros);
            c->weights.resize(kWeightBytes);
            PT_CUDA(cudaMemset(c->weights.get(), 0, kWeightBytes));
            c->ema_weights.resize(kWeightBytes);
            PT_CUDA(cudaMemset(c->ema_weights.get(), 0, kWeightBytes));
            c->ema.resize(kMasterFloats * sizeof(float));
            c->ctas = device_sm_count();
            c->partial.resize(size_t(c->ctas) * kMasterFloats * sizeof(float));
            c->loss_partial.resize(size_t(c->ctas) * sizeof(float));
            c->status.resize(sizeof(int));
            PT_CUDA(cudaMemset(c->status.get(), 0, sizeof(int)));
            c->step.resize(2 * sizeof(int));
            PT_CUDA(cudaMemset(c->step.get(), 0, 2 * sizeof(int)));
            c->done.resize(sizeof(unsigned));
            PT_CUDA(cudaMemset(c->done.get(), 0, sizeof(unsigned)));
            c->loss.resize(sizeof(float));
            PT_CUDA(cudaMemset(c->loss.get(), 0, sizeof(float)));
            PT_CUDA(cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kFwdSmem)));
            PT_CUDA(cudaFuncSetAttribute(train_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kTrainSmem)));
            refresh_canon(c, nullptr);
            PT_CUDA(cudaDeviceSynchronize());
        } catch (...) { delete c; throw; }
        *out = c;
    });
}

pt_status pt_cache_destroy(pt_cache *c) { delete c; return PT_OK; }

pt_status pt_cache_query_device(pt_cache *c, const pt_cache_query *queries, size_t count, float *rgb, void *stream) {
    return guard([&]() {
        if (!c || (count && (!queries || !rgb))) throw Error(PT_INVALID_ARGUMENT, "null argument");
        if (!count) return;
        cache_forward(c, queries, count, nullptr, rgb, static_cast<cudaStream_t>(stream));
    });
}

pt_status pt_cache_gradients(pt_cache *c, const pt_cache_query *queries, const float *targets, size_t count, float *grad_host,
                             float *loss) {
    return guard([&]() {
        if (!c || !queries || !targets || !count) throw Error(PT_INVALID_ARGUMENT, "invalid gradient arguments");
        gradients(c, queries, targets, count, nullptr, false, nullptr);
        float l = read_loss(c, nullptr);
        if (loss) *loss = l;
        if (grad_host) PT_CUDA(cudaMemcpy(grad_host, c->grad.get(), kMasterFloats * sizeof(float), cudaMemcpyDeviceToHost));
    });
}

pt_status pt_cache_train_device(pt_cache *c, const pt_cache_query *queries, const float *targets, size_t count, float *loss,
                                void *stream) {
    return guard([&]() {
        if (!c || !queries || !targets || !count) throw Error(PT_INVALID_ARGUMENT, "invalid training arguments");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        cache_train(c, queries, targets, count, nullptr, st);
        if (loss) *loss = read_loss(c, st);
    });
}

// Waits for `stream` and reports a timed-out tensor-core wait of an earlier call (clearing it).
pt_status pt_cache_sync(pt_cache *c, void *stream) {
    return guard([&]() {
        if (!c) throw Error(PT_INVALID_ARGUMENT, "null cache");
        PT_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
        check_status(c);
    });
}

// try_wait attempts per bounded tensor-core wait of this cache's kernels (< 0: the default).
pt_status pt_cache_wait_limit(pt_cache *c, long long attempts) {
    return guard([&]() {
        if (!c) throw Error(PT_INVALID_ARGUMENT, "null cache");
        c->attempts = attempts < 0 ? kSpinLimit : attempts;
    });
}

pt_status pt_cache_weights(pt_cache *c, float *get, const float *set, size_t floats) {
    return guard([&]() {
        if (!c || floats != size_t(kMasterFloats)) throw Error(PT_INVALID_ARGUMENT, "weights hold 20672 floats");
        if (get) PT_CUDA(cudaMemcpy(get, c->master.get(), floats * sizeof(float), cudaMemcpyDeviceToHost));
        if (set) {
            PT_CUDA(cudaMemcpy(c->master.get(), set, floats * sizeof(float), cudaMemcpyHostToDevice));
            refresh_canon(c, nullptr);
            PT_CUDA(cudaDeviceSynchronize());
        }
    });
}

pt_status pt_cache_average(pt_cache *c, float decay) {
    return guard([&]() {
        if (!c || !(decay >= 0 && decay < 1)) throw Error(PT_INVALID_ARGUMENT, "weight-average decay must be in [0, 1)");
        c->ema_decay = decay;
        PT_CUDA(cudaMemcpy(c->ema_weights.get(), c->weights.get(), kWeightBytes, cudaMemcpyDeviceToDevice));
        PT_CUDA(cudaMemset(c->ema.get(), 0, kMasterFloats * sizeof(float)));
        PT_CUDA(cudaMemset(c->step.get<int>() + 1, 0, sizeof(int)));
        PT_CUDA(cudaDeviceSynchronize());
    });
}

pt_status pt_cache_hyper(pt_cache *c, float lr, float beta1, float beta2, float eps) {
    return guard([&]() {
        if (!c || !(lr > 0) || !(beta1 >= 0 && beta1 < 1) || !(beta2 >= 0 && beta2 < 1) || !(eps > 0))
            throw Error(PT_INVALID_ARGUMENT, "invalid Adam settings");
        c->lr = lr; c->beta1 = beta1; c->beta2 = beta2; c->eps = eps;
    });
}

} // extern "C"
