// nps_oracle_mlp.cpp — CPU restatement of the learned-ADC policy network
// (test infrastructure; the product runs nprush_b200/csrc/mlp.cu).
//
// 16 -> 64 -> 64 -> 3 MLP with ReLU; softmax cross-entropy over
// {keep (logit 0), clone, split, prune}, weighted per class, averaged over the
// batch.  With round_bf16 the products take the operands the tensor-core
// kernel uses: weights, inputs, hidden activations and the back-propagated
// pre-activation gradients rounded to bf16 (round to nearest even), fp32
// sums, biases and bias gradients in fp32.  Without it everything stays in
// double, for central-difference checks of the backward.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {
constexpr int kIn = 16, kH = 64, kOut = 3;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kOut * kH, kNumParams = oB3 + kOut;

// IEEE binary32 -> bfloat16 -> binary32, round to nearest, ties to even
float bf16(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7F800000u) == 0x7F800000u) {  // inf / nan: truncate (keep nan quiet)
    if (u & 0x007FFFFFu) u |= 0x00400000u;
    u &= 0xFFFF0000u;
  } else {
    u += 0x7FFFu + ((u >> 16) & 1u);
    u &= 0xFFFF0000u;
  }
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

template <class T>
T rnd(T x, bool on) {
  return on ? (T)bf16((float)x) : x;
}

template <class T>
void run(const float* P, const float* X, const uint8_t* labels, uint32_t n, const float* cw, bool round_bf16,
         T* grads, T* loss, float* logits) {
  const bool r = round_bf16;
  std::vector<T> W(kNumParams);
  for (int i = 0; i < kNumParams; ++i) W[i] = (T)P[i];
  std::vector<T> Wb(W);
  for (int i = 0; i < kH * kIn; ++i) Wb[oW1 + i] = rnd(W[oW1 + i], r);
  for (int i = 0; i < kH * kH; ++i) Wb[oW2 + i] = rnd(W[oW2 + i], r);
  for (int i = 0; i < kOut * kH; ++i) Wb[oW3 + i] = rnd(W[oW3 + i], r);
  if (grads)
    for (int i = 0; i < kNumParams; ++i) grads[i] = 0;
  T L = 0;
  const T inv = (T)1 / (T)(n ? n : 1);
  for (uint32_t b = 0; b < n; ++b) {
    T x[kIn], h1[kH], h2[kH], z3[kOut];
    bool m1[kH], m2[kH];
    for (int k = 0; k < kIn; ++k) x[k] = rnd((T)X[(size_t)b * kIn + k], r);
    for (int o = 0; o < kH; ++o) {
      T s = 0;
      for (int k = 0; k < kIn; ++k) s += x[k] * Wb[oW1 + o * kIn + k];
      s += W[oB1 + o];
      m1[o] = s > 0;
      h1[o] = rnd(s > 0 ? s : (T)0, r);
    }
    for (int o = 0; o < kH; ++o) {
      T s = 0;
      for (int k = 0; k < kH; ++k) s += h1[k] * Wb[oW2 + o * kH + k];
      s += W[oB2 + o];
      m2[o] = s > 0;
      h2[o] = rnd(s > 0 ? s : (T)0, r);
    }
    for (int o = 0; o < kOut; ++o) {
      T s = 0;
      for (int k = 0; k < kH; ++k) s += h2[k] * Wb[oW3 + o * kH + k];
      z3[o] = s + W[oB3 + o];
      if (logits) logits[(size_t)b * kOut + o] = (float)z3[o];
    }
    if (!labels) continue;
    const uint32_t y = labels[b] & 3u;
    const T wy = (T)cw[y];
    const T zz[4] = {0, z3[0], z3[1], z3[2]};
    T m = zz[0];
    for (int k = 1; k < 4; ++k) m = zz[k] > m ? zz[k] : m;
    T e[4], se = 0;
    for (int k = 0; k < 4; ++k) se += (e[k] = std::exp(zz[k] - m));
    L += wy * (std::log(se) - (zz[y] - m)) * inv;
    if (!grads) continue;
    T d3[kOut], d3b[kOut];
    for (int k = 1; k < 4; ++k) d3[k - 1] = wy * (e[k] / se - (k == (int)y ? (T)1 : (T)0)) * inv;
    for (int k = 0; k < kOut; ++k) {
      d3b[k] = rnd(d3[k], r);
      grads[oB3 + k] += d3[k];
      for (int i = 0; i < kH; ++i) grads[oW3 + k * kH + i] += d3b[k] * h2[i];
    }
    T dz2b[kH];
    for (int i = 0; i < kH; ++i) {
      T s = 0;
      for (int k = 0; k < kOut; ++k) s += d3b[k] * Wb[oW3 + k * kH + i];
      const T dz = m2[i] ? s : (T)0;
      grads[oB2 + i] += dz;
      dz2b[i] = rnd(dz, r);
    }
    for (int o = 0; o < kH; ++o)
      for (int i = 0; i < kH; ++i) grads[oW2 + o * kH + i] += dz2b[o] * h1[i];
    for (int i = 0; i < kH; ++i) {
      T s = 0;
      for (int o = 0; o < kH; ++o) s += dz2b[o] * Wb[oW2 + o * kH + i];
      const T dz = m1[i] ? s : (T)0;
      grads[oB1 + i] += dz;
      const T dzb = rnd(dz, r);
      for (int k = 0; k < kIn; ++k) grads[oW1 + i * kIn + k] += dzb * x[k];
    }
  }
  if (loss) *loss = L;
}
}  // namespace

extern "C" {

int orc_mlp_num_params(void) { return kNumParams; }

// Gradients (kNumParams floats) and mean loss of one batch; logits (n x 3) if
// given.  labels may be null (forward only).
int orc_mlp_grads(const float* params, const float* X, const uint8_t* labels, uint32_t n, const float* class_w4,
                  int round_bf16, float* grads, float* loss, float* logits) {
  std::vector<float> g(kNumParams);
  float l = 0;
  run<float>(params, X, labels, n, class_w4, round_bf16 != 0, grads ? g.data() : nullptr, &l, logits);
  if (grads) std::memcpy(grads, g.data(), sizeof(float) * kNumParams);
  if (loss) *loss = l;
  return 0;
}

// Double precision, no rounding: loss and analytic gradients.
double orc_mlp_loss_f64(const float* params, const float* X, const uint8_t* labels, uint32_t n,
                        const float* class_w4, double* grads) {
  double l = 0;
  run<double>(params, X, labels, n, class_w4, false, grads, &l, nullptr);
  return l;
}
}
