// policy_net.cuh -- the precision-policy network shared by the tile policy
// (policy.cu) and the batched solver's chunk policy (batched.cu):
// 16 features -> 32 -> 32 -> 4 classes, ReLU, BF16 weights (held as float
// in shared memory), FP32 accumulation.
#pragma once

namespace mf {

constexpr int PN_NF = 16, PN_H1 = 32, PN_H2 = 32, PN_NO = 4;
constexpr int PN_OW1 = 0, PN_OB1 = PN_OW1 + PN_H1 * PN_NF, PN_OW2 = PN_OB1 + PN_H1, PN_OB2 = PN_OW2 + PN_H2 * PN_H1,
              PN_OW3 = PN_OB2 + PN_H2, PN_OB3 = PN_OW3 + PN_NO * PN_H2;
constexpr int PN_NPARAM = PN_OB3 + PN_NO;  // 1732
static_assert(PN_H1 == 32 && PN_H2 == 32, "one hidden unit per lane");

// One thread, the whole network.  Every unit starts from its bias and adds
// the products in input order with fused multiply-adds.
__device__ __forceinline__ void pn_forward(const float *w, const float *x, float *h1, float *h2, float *out)
{
    for (int j = 0; j < PN_H1; j++) {
        float s = w[PN_OB1 + j];
        for (int k = 0; k < PN_NF; k++) s = fmaf(w[PN_OW1 + j * PN_NF + k], x[k], s);
        h1[j] = fmaxf(s, 0.f);
    }
    for (int j = 0; j < PN_H2; j++) {
        float s = w[PN_OB2 + j];
        for (int k = 0; k < PN_H1; k++) s = fmaf(w[PN_OW2 + j * PN_H1 + k], h1[k], s);
        h2[j] = fmaxf(s, 0.f);
    }
    for (int o = 0; o < PN_NO; o++) {
        float s = w[PN_OB3 + o];
        for (int k = 0; k < PN_H2; k++) s = fmaf(w[PN_OW3 + o * PN_H2 + k], h2[k], s);
        out[o] = s;
    }
}

// One warp, the same operations in the same order: lane j computes hidden
// unit j of each layer, the inputs of the next layer come by shuffles, and
// every lane returns the four outputs.  All 32 lanes must call it.
__device__ __forceinline__ void pn_forward_warp(const float *w, const float *x, float *out)
{
    const int j = threadIdx.x & 31;
    float s = w[PN_OB1 + j];
    for (int k = 0; k < PN_NF; k++) s = fmaf(w[PN_OW1 + j * PN_NF + k], x[k], s);
    const float h1 = fmaxf(s, 0.f);
    s = w[PN_OB2 + j];
    for (int k = 0; k < PN_H1; k++) s = fmaf(w[PN_OW2 + j * PN_H1 + k], __shfl_sync(0xffffffffu, h1, k), s);
    const float h2 = fmaxf(s, 0.f);
    const int o = j & (PN_NO - 1);
    s = w[PN_OB3 + o];
    for (int k = 0; k < PN_H2; k++) s = fmaf(w[PN_OW3 + o * PN_H2 + k], __shfl_sync(0xffffffffu, h2, k), s);
    for (int k = 0; k < PN_NO; k++) out[k] = __shfl_sync(0xffffffffu, s, k);
}

}  // namespace mf
