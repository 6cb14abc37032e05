// microbench.cu -- integer-pipe throughput probes used as the roofline denominator.
//
// The scan is bound by integer issue, and the measured-peaks file of the pool carries only HBM
// and bf16 figures, so the INT32 peak is measured here, on the same device and clocks as the
// scan. Each probe runs independent dependency chains (8 per thread) of one instruction form
// over a full grid and reports lane operations per second. Kinds:
//   0 LOP3 (3-input logic)        1 IADD3 + LOP3 (2 adds, 1 xor) 2 IMAD (multiply-add)
//   3 POPC                        4 mixed generator step: IADD3 + LOP3 + IMAD + ISETP + VOTE
//   5 b1 tensor AND+POPC, mma.sync m16n8k256 (reported as 32-bit AND+POPC lane-ops: 1024 per mma)
//   6 SHF (funnel shift)          7 ISETP + VOTE + LOP3
//   8 generator step with the add issued as a multiply-add (IMAD + LOP3 + IMAD + ISETP + VOTE)
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kTpb = 256;
constexpr int kChains = 8;

template <int KIND>
__global__ void __launch_bounds__(kTpb) probe_kernel(uint32_t* sink, int iters, uint32_t k0, uint32_t k1) {
    uint32_t v[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) v[c] = threadIdx.x * 0x9E3779B9u + c * 0x85EBCA6Bu + blockIdx.x;
    uint32_t acc = 0;
    if constexpr (KIND == 5) {
        // Four independent accumulator sets so the probe measures throughput, not latency.
        int d[4][4] = {};
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int s = 0; s < 4; ++s)
                asm volatile(
                    "mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc "
                    "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                    : "+r"(d[s][0]), "+r"(d[s][1]), "+r"(d[s][2]), "+r"(d[s][3])
                    : "r"(v[s]), "r"(v[s + 1]), "r"(v[s + 2]), "r"(v[s + 3]), "r"(v[s + 4]), "r"(k0));
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) acc += (uint32_t)(d[s][0] + d[s][1] + d[s][2] + d[s][3]);
    } else {
        uint32_t bal[kChains] = {};
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int c = 0; c < kChains; ++c) {
                uint32_t x = v[c];
                if constexpr (KIND == 0) {
                    asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(x) : "r"(k0), "r"(k1));
                    asm volatile("lop3.b32 %0, %0, %1, %2, 0x78;" : "+r"(x) : "r"(k1), "r"(k0));
                } else if constexpr (KIND == 1) {
                    // Three-input adds whose operands change every step (no invariant folding).
                    const uint32_t y = v[(c + 1) % kChains], w = v[(c + 3) % kChains];
                    x = x + y + w;
                    x = x + w + (y ^ k0);
                } else if constexpr (KIND == 2) {
                    asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(k0), "r"(k1));
                    asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(k1), "r"(k0));
                } else if constexpr (KIND == 3) {
                    uint32_t y;
                    asm volatile("popc.b32 %0, %1;" : "=r"(y) : "r"(x));
                    asm volatile("popc.b32 %0, %1;" : "=r"(x) : "r"(y ^ k0));
                } else if constexpr (KIND == 4) {
                    // t = x + k0 + b; h = t ^ K; x = h * C + k1; b = ballot(x < T): 5 instructions,
                    // the ballot of one step feeding the add of the next.
                    asm volatile(
                        "{ .reg .pred p; .reg .u32 t, h;\n"
                        "add.u32 t, %0, %2; add.u32 t, t, %1;\n"
                        "xor.b32 h, t, 0x2F21A;\n"
                        "mad.lo.u32 %0, h, 0xC6D4F14B, %3;\n"
                        "setp.lt.u32 p, %0, 858993456;\n"
                        "vote.sync.ballot.b32 %1, p, 0xffffffff; }"
                        : "+r"(x), "+r"(bal[c])
                        : "r"(k0), "r"(k1));
                } else if constexpr (KIND == 7) {
                    // compare + ballot only
                    asm volatile(
                        "{ .reg .pred p;\n"
                        "setp.lt.u32 p, %0, %2;\n"
                        "vote.sync.ballot.b32 %1, p, 0xffffffff; }"
                        : "+r"(x), "+r"(bal[c])
                        : "r"(k0));
                    x ^= bal[c];
                } else if constexpr (KIND == 8) {
                    // generator step with the add as a multiply-add by a run-time 1 (k1 == 1 here)
                    asm volatile(
                        "{ .reg .pred p; .reg .u32 t, h;\n"
                        "mad.lo.u32 t, %1, %3, %0;\n"
                        "xor.b32 h, t, 0x2F21A;\n"
                        "mad.lo.u32 %0, h, 0xC6D4F14B, %2;\n"
                        "setp.lt.u32 p, %0, 858993456;\n"
                        "vote.sync.ballot.b32 %1, p, 0xffffffff; }"
                        : "+r"(x), "+r"(bal[c])
                        : "r"(k0), "r"(k1));
                } else if constexpr (KIND == 6) {
                    asm volatile("shf.r.wrap.b32 %0, %0, %1, %2;" : "+r"(x) : "r"(k0), "r"(k1));
                    asm volatile("shf.l.wrap.b32 %0, %1, %0, %2;" : "+r"(x) : "r"(k1), "r"(k0));
                }
                v[c] = x;
            }
        }
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc ^= v[c] ^ bal[c];
    }
    if (acc == 0x12345678u) sink[blockIdx.x] = acc;  // practically never taken; keeps the work
}

template <int KIND>
cudaError_t run(int blocks, int iters, float* ms) {
    uint32_t* sink = nullptr;
    cudaEvent_t a, b;
    cudaError_t e = cudaMalloc(&sink, blocks * sizeof(uint32_t));
    if (e != cudaSuccess) return e;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    probe_kernel<KIND><<<blocks, kTpb>>>(sink, iters / 8 + 1, 3u, 5u);  // warm-up
    cudaEventRecord(a);
    probe_kernel<KIND><<<blocks, kTpb>>>(sink, iters, 0x9E3779B9u, KIND == 8 ? 1u : 0x7F4A7C15u);
    cudaEventRecord(b);
    e = cudaEventSynchronize(b);
    cudaEventElapsedTime(ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace

extern "C" int32_t slime_b200_microbench(int32_t kind, int32_t iters, double* lane_ops_per_s, double* ms_out) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8;
    float ms = 0.f;
    cudaError_t e;
    double per_iter_thread;  // lane operations per thread per iteration
    switch (kind) {
        case 0: e = run<0>(blocks, iters, &ms); per_iter_thread = 2.0 * kChains; break;
        case 1: e = run<1>(blocks, iters, &ms); per_iter_thread = 3.0 * kChains; break;
        case 2: e = run<2>(blocks, iters, &ms); per_iter_thread = 2.0 * kChains; break;
        case 3: e = run<3>(blocks, iters, &ms); per_iter_thread = 2.0 * kChains; break;
        case 4: e = run<4>(blocks, iters, &ms); per_iter_thread = 5.0 * kChains; break;
        case 5: e = run<5>(blocks, iters, &ms); per_iter_thread = 4.0 * 1024.0 / 32.0; break;
        case 6: e = run<6>(blocks, iters, &ms); per_iter_thread = 2.0 * kChains; break;
        case 7: e = run<7>(blocks, iters, &ms); per_iter_thread = 3.0 * kChains; break;
        case 8: e = run<8>(blocks, iters, &ms); per_iter_thread = 5.0 * kChains; break;
        default: return -1;
    }
    if (e != cudaSuccess) return -1;
    const double ops = (double)blocks * kTpb * (double)iters * per_iter_thread;
    if (lane_ops_per_s) *lane_ops_per_s = ops / (ms * 1e-3);
    if (ms_out) *ms_out = ms;
    return 0;
}
