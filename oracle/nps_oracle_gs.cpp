// nps_oracle_gs.cpp — CPU oracle of the 3D Gaussian training model.
//
// TEST INFRASTRUCTURE ONLY (tests, smoke, and bench.py's CPU-baseline leg).
// The model has no counterpart in the reference (which fits generalised
// linear-parameter splats, splat_backward.wgsl:92-134); it is the model the
// library's Gaussian trainer implements, restated here independently of the
// CUDA code (the per-primitive math — SH basis, rotation, projection, split
// sampling — in gs_model.h, which includes nothing of the library):
//   * standard 3D Gaussians: mean, log-scales, quaternion, opacity logit,
//     real SH up to degree 3 (colour = SH + 0.5, clamped at 0);
//   * EWA projection with +0.3 px^2 low-pass; tile rectangle from the box of
//     the alpha >= 1/255 ellipse (Gaussians with 255 o <= 1 culled); tiles of
//     16x16, per-tile lists ordered by (f32 view depth, index);
//   * compositing with alpha = min(0.99, o * G), skip alpha < 1/255, stop
//     before T would fall below 1e-4;
//   * loss, by kind: 0 = (1 - l) mean|x - y| + l (1 - mean SSIM), 11x11
//     Gaussian window (sigma 1.5), zero padding, C1 = 0.01^2, C2 = 0.03^2,
//     l = 0.2 by default; 1 = mean|x - y|; 2 = mean (x - y)^2; means over the
//     3 H W V colour values.
// Two products:
//   orc_gs_forward / orc_gs_loss / orc_gs_backward / orc_gs_adam: the fp32
//     training step (also the timed CPU baseline, OpenMP over tiles);
//   orc_gs_loss_cd: FP64 central differences of the loss with the discrete
//     decisions (tile lists, skips, termination, clamps, |.| signs) frozen at
//     the base point, i.e. the derivative of the smooth piece the analytic
//     backward differentiates.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "gs_model.h"

using namespace orc_gm;

namespace {

constexpr double kLowpass = 0.3, kNear = 0.2, kAlphaMin = 1.0 / 255.0, kAlphaMax = 0.99, kTMin = 1e-4;
constexpr int kWin = 11;
// loss kinds (the library's NPS_GS_LOSS_* values)
constexpr int kLossL1Dssim = 0, kLossL1 = 1, kLossL2 = 2;

template <class T>
struct PreG {
  bool vis = false;
  T u, v, ca, cb, cc, op, col[3], depth;
  bool clamped[3];
  int x0, x1, y0, y1;
  float dkey;
};

template <class T>
void preprocess(const T* params, uint32_t n, int deg, const float* view, uint32_t W, uint32_t H,
                std::vector<PreG<T>>& out) {
  out.assign(n, PreG<T>());
  const uint32_t tx = (W + 15) / 16, ty = (H + 15) / 16;
  for (uint32_t i = 0; i < n; ++i) {
    const T* p = params + (size_t)i * kP;
    Footprint<T> P;
    project_gaussian<T>(view, p, (T)W, (T)H, (T)kLowpass, P);
    PreG<T>& g = out[i];
    // every field is filled even for culled Gaussians (frozen replays read them)
    g.u = P.u; g.v = P.v; g.ca = P.ca; g.cb = P.cb; g.cc = P.cc;
    g.depth = P.cw;
    g.dkey = (float)P.cw;
    g.op = (T)1 / ((T)1 + std::exp(-p[kOpacity]));
    const T dx = p[0] - (T)view[32], dy = p[1] - (T)view[33], dz = p[2] - (T)view[34];
    const T il = (T)1 / std::sqrt(std::max(dx * dx + dy * dy + dz * dz, (T)1e-20));
    T basis[16];
    real_sh<T>(deg, dx * il, dy * il, dz * il, basis);
    const int nb = (deg + 1) * (deg + 1);
    for (int c = 0; c < 3; ++c) {
      T col = (T)0.5;
      for (int k = 0; k < nb; ++k) col += basis[k] * p[kSH + 3 * k + c];
      g.clamped[c] = col < 0;
      g.col[c] = col < 0 ? (T)0 : col;
    }
    g.x0 = g.x1 = g.y0 = g.y1 = 0;
    // footprint: the alpha >= 1/255 ellipse d^T Sigma^-1 d <= 2 ln(255 o)
    // (1% margin), bounded by centre +- sqrt(t2 Sigma_xx), +- sqrt(t2 Sigma_yy)
    if (!(P.cw > (T)kNear && P.det > 0 && g.op * (T)255 > (T)1)) continue;
    const T t2 = (T)2 * std::log((T)255 * g.op) * (T)1.01;
    const T ex = std::sqrt(t2 * P.A), ey = std::sqrt(t2 * P.C);
    const int x0 = std::max(0, std::min((int)tx, (int)std::floor((P.u - ex) / (T)16)));
    const int x1 = std::max(0, std::min((int)tx, (int)std::floor((P.u + ex) / (T)16) + 1));
    const int y0 = std::max(0, std::min((int)ty, (int)std::floor((P.v - ey) / (T)16)));
    const int y1 = std::max(0, std::min((int)ty, (int)std::floor((P.v + ey) / (T)16) + 1));
    if (!(x1 > x0 && y1 > y0)) continue;
    g.vis = true;
    g.x0 = x0; g.x1 = x1; g.y0 = y0; g.y1 = y1;
  }
}

template <class T>
std::vector<std::vector<uint32_t>> tile_lists(const std::vector<PreG<T>>& pre, uint32_t W, uint32_t H) {
  const uint32_t tx = (W + 15) / 16, ty = (H + 15) / 16;
  std::vector<std::vector<uint32_t>> lists((size_t)tx * ty);
  for (uint32_t i = 0; i < pre.size(); ++i) {
    const PreG<T>& g = pre[i];
    if (!g.vis) continue;
    for (int y = g.y0; y < g.y1; ++y)
      for (int x = g.x0; x < g.x1; ++x) lists[(size_t)y * tx + x].push_back(i);
  }
  for (auto& l : lists)
    std::stable_sort(l.begin(), l.end(), [&](uint32_t a, uint32_t b) { return pre[a].dkey < pre[b].dkey; });
  return lists;
}

// Per-pixel record of the discrete decisions at the base point.
struct Frozen {
  std::vector<std::vector<uint32_t>> contrib;   // per (view, pixel): Gaussians that contributed, front to back
  std::vector<std::vector<uint8_t>> clamped;    // alpha clamped at 0.99
  std::vector<std::vector<uint8_t>> colclamp;   // per view: 3 flags per Gaussian
  std::vector<int8_t> l1sign;                   // per (view, pixel, channel)
};

std::vector<double> ssim_window() {
  std::vector<double> w(kWin);
  double s = 0;
  for (int k = 0; k < kWin; ++k) {
    double d = k - kWin / 2;
    w[k] = (float)std::exp(-d * d / (2.0 * 1.5 * 1.5));
    s += w[k];
  }
  for (int k = 0; k < kWin; ++k) w[k] = (float)(w[k] / s);
  return w;
}

// separable correlation with zero padding
template <class T>
void conv2(const T* in, T* out, uint32_t W, uint32_t H, const std::vector<double>& w) {
  std::vector<T> tmp((size_t)W * H);
  const int r = kWin / 2;
  for (uint32_t y = 0; y < H; ++y)
    for (uint32_t x = 0; x < W; ++x) {
      T a = 0;
      for (int k = 0; k < kWin; ++k) {
        int xx = (int)x + k - r;
        if (xx >= 0 && xx < (int)W) a += (T)w[k] * in[(size_t)y * W + xx];
      }
      tmp[(size_t)y * W + x] = a;
    }
  for (uint32_t y = 0; y < H; ++y)
    for (uint32_t x = 0; x < W; ++x) {
      T a = 0;
      for (int k = 0; k < kWin; ++k) {
        int yy = (int)y + k - r;
        if (yy >= 0 && yy < (int)H) a += (T)w[k] * tmp[(size_t)yy * W + x];
      }
      out[(size_t)y * W + x] = a;
    }
}

// loss of one view (sum of |x-y| and of SSIM over 3HW) and, optionally, the
// per-pixel derivative maps (dL/dx = conv(P1) + 2 x conv(P2) + y conv(P3))
template <class T>
void ssim_terms(const T* x3, const float* y4, uint32_t W, uint32_t H, T* l1_sum, T* ssim_sum,
                std::vector<T>* P123 /* 9 * W * H or null */, T dLds, const int8_t* sign_frozen) {
  const auto w = ssim_window();
  const size_t np = (size_t)W * H;
  std::vector<T> xc(np), yc(np), xx(np), yy(np), xy(np), mx(np), my(np), exx(np), eyy(np), exy(np);
  const T C1 = (T)(0.01 * 0.01), C2 = (T)(0.03 * 0.03);
  // the sums over every pixel accumulate in double (a float running sum over
  // an 800 x 800 view drifts by ~1e-4 relative)
  double l1_acc = 0.0, ssim_acc = 0.0;
  if (P123) P123->assign(9 * np, 0);
  for (int c = 0; c < 3; ++c) {
    for (size_t i = 0; i < np; ++i) {
      xc[i] = x3[3 * i + c];
      yc[i] = (T)y4[4 * i + c];
      xx[i] = xc[i] * xc[i];
      yy[i] = yc[i] * yc[i];
      xy[i] = xc[i] * yc[i];
      const T d = xc[i] - yc[i];
      if (sign_frozen)
        l1_acc += (double)((T)sign_frozen[3 * i + c] * d);
      else
        l1_acc += (double)(d < 0 ? -d : d);
    }
    conv2(xc.data(), mx.data(), W, H, w);
    conv2(yc.data(), my.data(), W, H, w);
    conv2(xx.data(), exx.data(), W, H, w);
    conv2(yy.data(), eyy.data(), W, H, w);
    conv2(xy.data(), exy.data(), W, H, w);
    for (size_t i = 0; i < np; ++i) {
      const T sxx = exx[i] - mx[i] * mx[i], syy = eyy[i] - my[i] * my[i], sxy = exy[i] - mx[i] * my[i];
      const T A1 = 2 * mx[i] * my[i] + C1, A2 = 2 * sxy + C2, B1 = mx[i] * mx[i] + my[i] * my[i] + C1,
              B2 = sxx + syy + C2;
      const T s = (A1 * A2) / (B1 * B2);
      ssim_acc += (double)s;
      if (P123) {
        const T ds_dmx = (2 * my[i] * A2) / (B1 * B2) - s * 2 * mx[i] / B1;
        const T ds_dsxx = -s / B2, ds_dsxy = 2 * A1 / (B1 * B2);
        const T dm = dLds * ds_dmx, d2 = dLds * ds_dsxx, dxy = dLds * ds_dsxy;
        (*P123)[9 * i + 3 * c + 0] = dm - 2 * mx[i] * d2 - my[i] * dxy;
        (*P123)[9 * i + 3 * c + 1] = d2;
        (*P123)[9 * i + 3 * c + 2] = dxy;
      }
    }
  }
  *l1_sum = (T)l1_acc;
  *ssim_sum = (T)ssim_acc;
}

// Render one view.  Record mode (frz != null, replay == false) stores the
// decisions; replay mode composites exactly the recorded contributors.
template <class T>
void render_view(const T* params, uint32_t n, int deg, const float* view, uint32_t W, uint32_t H, const float* bg,
                 uint32_t vidx, T* img3, T* Tfin, uint32_t* ncontrib, Frozen* frz, bool replay) {
  std::vector<PreG<T>> pre;
  preprocess<T>(params, n, deg, view, W, H, pre);
  const uint32_t tx = (W + 15) / 16;
  const size_t np = (size_t)W * H;
  if (frz && !replay) {
    frz->colclamp.resize(std::max<size_t>(frz->colclamp.size(), vidx + 1));
    frz->colclamp[vidx].assign(3 * (size_t)n, 0);
    for (uint32_t i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c) frz->colclamp[vidx][3 * i + c] = pre[i].vis && pre[i].clamped[c];
  }
  if (replay) {
    // colour clamps as at the base point
    for (uint32_t i = 0; i < n; ++i)
      for (int c = 0; c < 3; ++c)
        if (frz->colclamp[vidx][3 * i + c]) pre[i].col[c] = 0;
        else if (pre[i].clamped[c]) {
          // recompute the unclamped colour (the perturbation crossed zero)
          const T* p = params + (size_t)i * kP;
          const T dx = p[0] - (T)view[32], dy = p[1] - (T)view[33], dz = p[2] - (T)view[34];
          const T il = (T)1 / std::sqrt(std::max(dx * dx + dy * dy + dz * dz, (T)1e-20));
          T basis[16];
          real_sh<T>(deg, dx * il, dy * il, dz * il, basis);
          T col = (T)0.5;
          for (int k = 0; k < (deg + 1) * (deg + 1); ++k) col += basis[k] * p[kSH + 3 * k + c];
          pre[i].col[c] = col;
        }
    for (size_t pix = 0; pix < np; ++pix) {
      const uint32_t px = pix % W, py = pix / W;
      const auto& lst = frz->contrib[(size_t)vidx * np + pix];
      const auto& clp = frz->clamped[(size_t)vidx * np + pix];
      T Tt = 1, C[3] = {0, 0, 0};
      for (size_t k = 0; k < lst.size(); ++k) {
        const PreG<T>& g = pre[lst[k]];
        const T dx = g.u - (T)px, dy = g.v - (T)py;
        const T power = (T)-0.5 * (g.ca * dx * dx + g.cc * dy * dy) - g.cb * dx * dy;
        const T alpha = clp[k] ? (T)kAlphaMax : g.op * std::exp(power);
        for (int c = 0; c < 3; ++c) C[c] += g.col[c] * alpha * Tt;
        Tt = Tt * (1 - alpha);
      }
      for (int c = 0; c < 3; ++c) img3[3 * pix + c] = C[c] + Tt * (T)bg[c];
      if (Tfin) Tfin[pix] = Tt;
    }
    return;
  }
  const auto lists = tile_lists<T>(pre, W, H);
  if (frz) {
    const size_t need = (size_t)(vidx + 1) * np;
    if (frz->contrib.size() < need) {
      frz->contrib.resize(need);
      frz->clamped.resize(need);
    }
  }
#pragma omp parallel for schedule(dynamic, 4) if (!frz)
  for (long pixl = 0; pixl < (long)np; ++pixl) {
    const size_t pix = (size_t)pixl;
    const uint32_t px = pix % W, py = pix / W;
    const auto& lst = lists[(size_t)(py / 16) * tx + px / 16];
    T Tt = 1, C[3] = {0, 0, 0};
    uint32_t last = 0;
    std::vector<uint32_t>* rc = frz ? &frz->contrib[(size_t)vidx * np + pix] : nullptr;
    std::vector<uint8_t>* rk = frz ? &frz->clamped[(size_t)vidx * np + pix] : nullptr;
    if (rc) { rc->clear(); rk->clear(); }
    for (size_t k = 0; k < lst.size(); ++k) {
      const PreG<T>& g = pre[lst[k]];
      const T dx = g.u - (T)px, dy = g.v - (T)py;
      const T power = (T)-0.5 * (g.ca * dx * dx + g.cc * dy * dy) - g.cb * dx * dy;
      if (power > 0) continue;
      const T araw = g.op * std::exp(power);
      const T alpha = std::min((T)kAlphaMax, araw);
      if (alpha < (T)kAlphaMin) continue;
      const T test_T = Tt * (1 - alpha);
      if (test_T < (T)kTMin) break;
      for (int c = 0; c < 3; ++c) C[c] += g.col[c] * alpha * Tt;
      Tt = test_T;
      last = (uint32_t)k + 1;
      if (rc) { rc->push_back(lst[k]); rk->push_back(araw > (T)kAlphaMax); }
    }
    for (int c = 0; c < 3; ++c) img3[3 * pix + c] = C[c] + Tt * (T)bg[c];
    if (Tfin) Tfin[pix] = Tt;
    if (ncontrib) ncontrib[pix] = last;
  }
}

template <class T>
T total_loss(const T* params, uint32_t n, int deg, const float* views, uint32_t nv, uint32_t W, uint32_t H,
             const float* bg, const float* tgt_all, const uint32_t* tids, double lambda, int kind, Frozen* frz,
             bool replay) {
  const size_t np = (size_t)W * H;
  std::vector<T> img(3 * np);
  T l1 = 0, ss = 0, sq = 0;  // per-view sums added once each (the pixel sums run in double below)
  if (frz && !replay) frz->l1sign.assign(3 * np * nv, 0);
  for (uint32_t v = 0; v < nv; ++v) {
    render_view<T>(params, n, deg, views + (size_t)kViewRec * v, W, H, bg, v, img.data(), nullptr, nullptr, frz,
                   replay);
    const float* y4 = tgt_all + (size_t)tids[v] * np * 4;
    if (frz && !replay)
      for (size_t i = 0; i < np; ++i)
        for (int c = 0; c < 3; ++c) {
          T d = img[3 * i + c] - (T)y4[4 * i + c];
          frz->l1sign[(size_t)v * 3 * np + 3 * i + c] = d > 0 ? 1 : (d < 0 ? -1 : 0);
        }
    if (kind == kLossL2) {
      double acc = 0.0;
      for (size_t i = 0; i < np; ++i)
        for (int c = 0; c < 3; ++c) {
          const T d = img[3 * i + c] - (T)y4[4 * i + c];
          acc += (double)(d * d);
        }
      sq += (T)acc;
      continue;
    }
    if (kind == kLossL1) {
      const int8_t* sg = (frz && replay) ? &frz->l1sign[(size_t)v * 3 * np] : nullptr;
      double acc = 0.0;
      for (size_t i = 0; i < np; ++i)
        for (int c = 0; c < 3; ++c) {
          const T d = img[3 * i + c] - (T)y4[4 * i + c];
          acc += (double)(sg ? (T)sg[3 * i + c] * d : (d < 0 ? -d : d));
        }
      l1 += (T)acc;
      continue;
    }
    T a, b;
    ssim_terms<T>(img.data(), y4, W, H, &a, &b, nullptr, 0,
                  (frz && replay) ? &frz->l1sign[(size_t)v * 3 * np] : nullptr);
    l1 += a;
    ss += b;
  }
  const T inv = (T)1 / ((T)3 * (T)np * (T)nv);
  if (kind == kLossL2) return sq * inv;
  if (kind == kLossL1) return l1 * inv;
  return ((T)1 - (T)lambda) * l1 * inv + (T)lambda * ((T)1 - ss * inv);
}

}  // namespace

extern "C" {

// FP64 probes of the model's building blocks, for checks of gs_model.h on
// its own terms.  SH basis of degree 3 and its partials at n directions
// (dirs n x 3; each output n x 16).
int orc_gs_sh(const double* dirs, uint32_t n, double* b, double* gx, double* gy, double* gz) {
  for (uint32_t i = 0; i < n; ++i) {
    const double* d = dirs + 3 * (size_t)i;
    real_sh<double>(3, d[0], d[1], d[2], b + 16 * (size_t)i);
    real_sh_grad<double>(3, d[0], d[1], d[2], gx + 16 * (size_t)i, gy + 16 * (size_t)i, gz + 16 * (size_t)i);
  }
  return 0;
}

// Rotation of the unit quaternion q (R 9, row-major) and the vector-Jacobian
// product dq = sum G[r][c] dR[r][c]/dq (G 9, dq 4).
int orc_gs_rot(const double* q, const double* G9, double* R9, double* dq) {
  double R[3][3], G[3][3];
  for (int k = 0; k < 9; ++k) G[k / 3][k % 3] = G9[k];
  quat_rotation<double>(q[0], q[1], q[2], q[3], R);
  for (int k = 0; k < 9; ++k) R9[k] = R[k / 3][k % 3];
  quat_rotation_vjp<double>(q[0], q[1], q[2], q[3], G, dq);
  return 0;
}

// fp32 forward of V views: img V x H x W x 4 (rgb, final T), ncontrib V x H x W
int orc_gs_forward(const float* params, uint32_t n, int deg, const float* views, uint32_t nv, uint32_t W, uint32_t H,
                   const float* bg, float* img, uint32_t* ncontrib) {
  const size_t np = (size_t)W * H;
  std::vector<float> im3(3 * np), Tf(np);
  for (uint32_t v = 0; v < nv; ++v) {
    render_view<float>(params, n, deg, views + (size_t)kViewRec * v, W, H, bg, v, im3.data(), Tf.data(),
                       ncontrib + (size_t)v * np, nullptr, false);
    for (size_t i = 0; i < np; ++i) {
      float* o = img + ((size_t)v * np + i) * 4;
      o[0] = im3[3 * i]; o[1] = im3[3 * i + 1]; o[2] = im3[3 * i + 2]; o[3] = Tf[i];
    }
  }
  return 0;
}

// fp32 loss and dL/dimage (V x H x W x 4, alpha channel 0).  loss3 =
// (loss, mean |x - y|, mean SSIM) for kind 0, (loss, mean |x - y|, mean
// (x - y)^2) for kinds 1 and 2.
int orc_gs_loss(const float* img, const float* tgt_all, const uint32_t* tids, uint32_t nv, uint32_t W, uint32_t H,
                float lambda, int kind, float* loss3, float* dimg) {
  const size_t np = (size_t)W * H;
  const auto w = ssim_window();
  const float inv = (float)(1.0 / (3.0 * (double)np * nv));
  double l1 = 0, ss = 0, sq = 0;
  std::vector<float> x3(3 * np), P, c1(np), c2(np), c3(np), tmp(np);
  for (uint32_t v = 0; v < nv; ++v) {
    for (size_t i = 0; i < np; ++i)
      for (int c = 0; c < 3; ++c) x3[3 * i + c] = img[((size_t)v * np + i) * 4 + c];
    const float* y4 = tgt_all + (size_t)tids[v] * np * 4;
    if (kind != kLossL1Dssim) {
      for (size_t i = 0; i < np; ++i) {
        for (int c = 0; c < 3; ++c) {
          const float d = x3[3 * i + c] - y4[4 * i + c];
          l1 += std::fabs(d);
          sq += (double)d * d;
          if (dimg) {
            const float sgn = d > 0 ? 1.0f : (d < 0 ? -1.0f : 0.0f);
            dimg[((size_t)v * np + i) * 4 + c] = kind == kLossL2 ? 2.0f * d * inv : sgn * inv;
          }
        }
        if (dimg) dimg[((size_t)v * np + i) * 4 + 3] = 0.0f;
      }
      continue;
    }
    float a, b;
    ssim_terms<float>(x3.data(), y4, W, H, &a, &b, &P, -lambda * inv, nullptr);
    l1 += a;
    ss += b;
    if (!dimg) continue;
    for (int c = 0; c < 3; ++c) {
      for (int q = 0; q < 3; ++q) {
        for (size_t i = 0; i < np; ++i) tmp[i] = P[9 * i + 3 * c + q];
        conv2(tmp.data(), q == 0 ? c1.data() : q == 1 ? c2.data() : c3.data(), W, H, w);
      }
      for (size_t i = 0; i < np; ++i) {
        const float x = x3[3 * i + c], y = y4[4 * i + c];
        const float d = x - y;
        const float sgn = d > 0 ? 1.0f : (d < 0 ? -1.0f : 0.0f);
        dimg[((size_t)v * np + i) * 4 + c] = c1[i] + 2.0f * x * c2[i] + y * c3[i] + (1.0f - lambda) * inv * sgn;
      }
    }
    for (size_t i = 0; i < np; ++i) dimg[((size_t)v * np + i) * 4 + 3] = 0.0f;
  }
  if (loss3) {
    if (kind == kLossL1Dssim) {
      loss3[0] = (float)((1.0 - lambda) * l1 * inv + lambda * (1.0 - ss * inv));
      loss3[2] = (float)(ss * inv);
    } else {
      loss3[0] = (float)((kind == kLossL2 ? sq : l1) * inv);
      loss3[2] = (float)(sq * inv);
    }
    loss3[1] = (float)(l1 * inv);
  }
  return 0;
}

// fp32 backward: screen-space gradients per (view, Gaussian) by reverse
// traversal from the final T, then the projection chain summed over views.
// grads: n x 64 (overwritten).
// adc2 (optional, n x 2): += (sum over the views that see a Gaussian of the
// NDC-space norm of d(view loss)/d(mean2D), number of those views), where the
// view loss is the given loss times adc_scale (the views it averages over).
int orc_gs_backward(const float* params, uint32_t n, int deg, const float* views, uint32_t nv, uint32_t W, uint32_t H,
                    const float* bg, const float* img, const uint32_t* ncontrib, const float* dimg, float* grads,
                    float* adc2, float adc_scale) {
  const size_t np = (size_t)W * H;
  const uint32_t tx = (W + 15) / 16;
  std::vector<float> g2((size_t)nv * n * 10, 0.0f);
  std::vector<std::vector<PreG<float>>> pres(nv);
  for (uint32_t v = 0; v < nv; ++v) {
    const float* view = views + (size_t)kViewRec * v;
    std::vector<PreG<float>>& pre = pres[v];
    preprocess<float>(params, n, deg, view, W, H, pre);
    const auto lists = tile_lists<float>(pre, W, H);
    float* gv = &g2[(size_t)v * n * 10];
    const uint32_t ntiles = (uint32_t)lists.size();
#pragma omp parallel
    {
      std::vector<float> local((size_t)n * 10, 0.0f);
      std::vector<uint8_t> touched(n, 0);
#pragma omp for schedule(dynamic, 2)
      for (long t = 0; t < (long)ntiles; ++t) {
        const auto& lst = lists[t];
        const uint32_t x0 = (uint32_t)(t % tx) * 16, y0 = (uint32_t)(t / tx) * 16;
        for (uint32_t py = y0; py < std::min(y0 + 16, H); ++py)
          for (uint32_t px = x0; px < std::min(x0 + 16, W); ++px) {
            const size_t pix = (size_t)py * W + px;
            const float* o = img + ((size_t)v * np + pix) * 4;
            const float* d = dimg + ((size_t)v * np + pix) * 4;
            float T = o[3];
            const float T_final = o[3];
            const uint32_t last = ncontrib[(size_t)v * np + pix];
            const float dC[3] = {d[0], d[1], d[2]};
            const float bg_dot = bg[0] * dC[0] + bg[1] * dC[1] + bg[2] * dC[2];
            float accum[3] = {0, 0, 0}, last_col[3] = {0, 0, 0}, last_alpha = 0;
            for (int k = (int)last - 1; k >= 0; --k) {
              const uint32_t gi = lst[k];
              const PreG<float>& g = pre[gi];
              const float dx = g.u - (float)px, dy = g.v - (float)py;
              const float power = -0.5f * (g.ca * dx * dx + g.cc * dy * dy) - g.cb * dx * dy;
              if (power > 0) continue;
              const float G = std::exp(power);
              const float araw = g.op * G;
              const float alpha = std::min((float)kAlphaMax, araw);
              if (alpha < (float)kAlphaMin) continue;
              T = T / (1.0f - alpha);
              const float wgt = alpha * T;
              float dL_dalpha = 0;
              float* L = &local[(size_t)gi * 10];
              for (int c = 0; c < 3; ++c) {
                accum[c] = last_alpha * last_col[c] + (1.0f - last_alpha) * accum[c];
                last_col[c] = g.col[c];
                dL_dalpha += (g.col[c] - accum[c]) * dC[c];
                L[6 + c] += wgt * dC[c];
              }
              dL_dalpha *= T;
              last_alpha = alpha;
              dL_dalpha += (-T_final / (1.0f - alpha)) * bg_dot;
              if (araw <= (float)kAlphaMax) {
                const float dL_dG = g.op * dL_dalpha;
                const float gdx = G * dx, gdy = G * dy;
                L[0] += dL_dG * (-gdx * g.ca - gdy * g.cb);
                L[1] += dL_dG * (-gdy * g.cc - gdx * g.cb);
                L[2] += -0.5f * gdx * dx * dL_dG;
                L[3] += -gdx * dy * dL_dG;
                L[4] += -0.5f * gdy * dy * dL_dG;
                L[5] += G * dL_dalpha;
              }
              touched[gi] = 1;
            }
          }
      }
#pragma omp critical
      for (uint32_t i = 0; i < n; ++i)
        if (touched[i])
          for (int k = 0; k < 10; ++k) gv[(size_t)i * 10 + k] += local[(size_t)i * 10 + k];
    }
  }
#pragma omp parallel for schedule(static)
  for (long il = 0; il < (long)n; ++il) {
    const uint32_t i = (uint32_t)il;
    const float* p = params + (size_t)i * kP;
    float gm[3] = {0, 0, 0}, gls[3] = {0, 0, 0}, gq[4] = {0, 0, 0, 0}, gop = 0, gsh[48] = {0};
    const int nb = (deg + 1) * (deg + 1);
    const float op = 1.0f / (1.0f + std::exp(-p[kOpacity]));
    for (uint32_t v = 0; v < nv; ++v) {
      const PreG<float>& pg = pres[v][i];
      if (!pg.vis) continue;
      const float* gr = &g2[((size_t)v * n + i) * 10];
      const float* view = views + (size_t)kViewRec * v;
      Footprint<float> P;
      project_gaussian<float>(view, p, (float)W, (float)H, (float)kLowpass, P);
      gop += gr[5];
      if (adc2) {
        const float du = gr[0] * 0.5f * (float)W, dv = gr[1] * 0.5f * (float)H;
        adc2[2 * (size_t)i] += adc_scale * std::sqrt(du * du + dv * dv);
        adc2[2 * (size_t)i + 1] += 1.0f;
      }
      float dc[3];
      for (int c = 0; c < 3; ++c) dc[c] = pg.clamped[c] ? 0.0f : gr[6 + c];
      const float ddx = p[0] - view[32], ddy = p[1] - view[33], ddz = p[2] - view[34];
      const float il2 = 1.0f / std::sqrt(std::max(ddx * ddx + ddy * ddy + ddz * ddz, 1e-20f));
      const float dir[3] = {ddx * il2, ddy * il2, ddz * il2};
      float basis[16];
      real_sh<float>(deg, dir[0], dir[1], dir[2], basis);
      if (deg > 0) {
        float bx[16], by[16], bz[16], ddir[3] = {0, 0, 0};
        real_sh_grad<float>(deg, dir[0], dir[1], dir[2], bx, by, bz);
        for (int k = 1; k < nb; ++k) {
          const float s = p[kSH + 3 * k] * dc[0] + p[kSH + 3 * k + 1] * dc[1] + p[kSH + 3 * k + 2] * dc[2];
          ddir[0] += s * bx[k]; ddir[1] += s * by[k]; ddir[2] += s * bz[k];
        }
        const float dd = dir[0] * ddir[0] + dir[1] * ddir[1] + dir[2] * ddir[2];
        for (int c = 0; c < 3; ++c) gm[c] += (ddir[c] - dir[c] * dd) * il2;
      }
      for (int k = 0; k < nb; ++k)
        for (int c = 0; c < 3; ++c) gsh[3 * k + c] += basis[k] * dc[c];
      // conic -> covariance
      const float ia = P.ca, ib = P.cb, ic = P.cc;
      const float h00 = gr[2], h01 = 0.5f * gr[3], h11 = gr[4];
      const float x00 = h00 * ia + h01 * ib, x01 = h00 * ib + h01 * ic, x10 = h01 * ia + h11 * ib,
                  x11 = h01 * ib + h11 * ic;
      const float G00 = -(ia * x00 + ib * x10), G01 = -(ia * x01 + ib * x11), G10 = -(ib * x00 + ic * x10),
                  G11 = -(ib * x01 + ic * x11);
      const float Gs[2][2] = {{G00, 0.5f * (G01 + G10)}, {0.5f * (G01 + G10), G11}};
      float GJ[2][3], dS[3][3], dJ[2][3];
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c) GJ[r][c] = Gs[r][0] * P.J[0][c] + Gs[r][1] * P.J[1][c];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) dS[r][c] = P.J[0][r] * GJ[0][c] + P.J[1][r] * GJ[1][c];
      for (int r = 0; r < 2; ++r)
        for (int c = 0; c < 3; ++c) dJ[r][c] = 2.0f * (GJ[r][0] * P.S[0][c] + GJ[r][1] * P.S[1][c] + GJ[r][2] * P.S[2][c]);
      const float r0[3] = {view[0], view[4], view[8]}, r1[3] = {view[1], view[5], view[9]},
                  r3[3] = {view[3], view[7], view[11]};
      const float a = 0.5f * W, b = 0.5f * H, iw = 1.0f / P.cw, iw2 = iw * iw, iw3 = iw2 * iw;
      const float d0r0 = dJ[0][0] * r0[0] + dJ[0][1] * r0[1] + dJ[0][2] * r0[2];
      const float d0r3 = dJ[0][0] * r3[0] + dJ[0][1] * r3[1] + dJ[0][2] * r3[2];
      const float d1r1 = dJ[1][0] * r1[0] + dJ[1][1] * r1[1] + dJ[1][2] * r1[2];
      const float d1r3 = dJ[1][0] * r3[0] + dJ[1][1] * r3[1] + dJ[1][2] * r3[2];
      for (int l = 0; l < 3; ++l) {
        gm[l] += a * (-d0r0 * r3[l] * iw2 - d0r3 * r0[l] * iw2 + 2.0f * P.cx * d0r3 * r3[l] * iw3);
        gm[l] += -b * (-d1r1 * r3[l] * iw2 - d1r3 * r1[l] * iw2 + 2.0f * P.cy * d1r3 * r3[l] * iw3);
        gm[l] += P.J[0][l] * gr[0] + P.J[1][l] * gr[1];
      }
      float dM[3][3], dR[3][3];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) dM[r][c] = 2.0f * (dS[r][0] * P.M[0][c] + dS[r][1] * P.M[1][c] + dS[r][2] * P.M[2][c]);
      for (int c = 0; c < 3; ++c) {
        float ds = 0;
        for (int r = 0; r < 3; ++r) {
          ds += dM[r][c] * P.R[r][c];
          dR[r][c] = dM[r][c] * P.sc[c];
        }
        gls[c] += ds * P.sc[c];
      }
      float dqn[4];
      quat_rotation_vjp<float>(P.qn[0], P.qn[1], P.qn[2], P.qn[3], dR, dqn);
      const float qd = P.qn[0] * dqn[0] + P.qn[1] * dqn[1] + P.qn[2] * dqn[2] + P.qn[3] * dqn[3];
      for (int k = 0; k < 4; ++k) gq[k] += (dqn[k] - P.qn[k] * qd) / P.qlen;
    }
    float* out = grads + (size_t)i * kP;
    std::memset(out, 0, sizeof(float) * kP);
    for (int k = 0; k < 3; ++k) { out[k] = gm[k]; out[3 + k] = gls[k]; }
    for (int k = 0; k < 4; ++k) out[6 + k] = gq[k];
    out[10] = gop * op * (1.0f - op);
    for (int k = 0; k < 48; ++k) out[kSH + k] = gsh[k];
  }
  return 0;
}

// Adam over the 59 used floats of each record (eps 1e-15, betas 0.9 / 0.999).
int orc_gs_adam(float* params, const float* grads, float* m, float* v, uint32_t n, uint32_t step, const float* lr6) {
  const float bc1 = (float)(1.0 - std::pow(0.9, (double)step)), bc2 = (float)(1.0 - std::pow(0.999, (double)step));
#pragma omp parallel for schedule(static)
  for (long il = 0; il < (long)n; ++il) {
    for (int k = 0; k < kUsed; ++k) {
      if (k == 11) continue;
      const size_t j = (size_t)il * kP + k;
      const float lr = k < 3 ? lr6[0] : k < 6 ? lr6[1] : k < 10 ? lr6[2] : k < 12 ? lr6[3] : k < 15 ? lr6[4] : lr6[5];
      const float g = grads[j];
      m[j] = 0.9f * m[j] + (1.0f - 0.9f) * g;
      v[j] = 0.999f * v[j] + (1.0f - 0.999f) * g * g;
      const float mh = m[j] / bc1, vh = v[j] / bc2;
      params[j] -= lr * mh / (std::sqrt(vh) + 1e-15f);
    }
  }
  return 0;
}

// Plain threshold ADC, serial: prune opacity < prune_op; densify (avg grad >=
// thresh) by split (max scale > split_scale) or clone, densifying candidates in
// index order while the capacity allows; records are compacted in index order,
// each parent's outputs in place of it.  Split children come from
// split_child (gs_model.h); clones keep the parent's Adam state in the first copy.
int orc_gs_adc(const float* params, const float* m, const float* v, const float* adc_grad, const float* adc_denom,
               uint32_t n, uint32_t cap, float thresh, float split_scale, float prune_op, uint32_t seed,
               float* out_p, float* out_m, float* out_v, uint32_t* counts4) {
  std::vector<uint32_t> flag(n);
  uint32_t kept = 0, cands = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const float* P = params + (size_t)i * kP;
    const float op = 1.0f / (1.0f + std::exp(-P[kOpacity]));
    uint32_t f = 0;
    if (!(op < prune_op)) {
      f = 1;
      const float d = adc_denom[i];
      const float avg = d > 0.0f ? adc_grad[i] / d : 0.0f;
      if (avg >= thresh) {
        f |= 2;
        if (std::exp(std::max(std::max(P[3], P[4]), P[5])) > split_scale) f |= 4;
      }
    }
    flag[i] = f;
    kept += f & 1;
    cands += (f >> 1) & 1;
  }
  const uint32_t budget = cap > kept ? cap - kept : 0;
  uint32_t o = 0, rank = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint32_t f = flag[i];
    if (!(f & 1)) continue;
    const bool dens = (f & 2) && rank < budget;
    if (f & 2) ++rank;
    const float* P = params + (size_t)i * kP;
    const size_t src = (size_t)i * kP;
    if (!dens) {
      std::copy(P, P + kP, out_p + (size_t)o * kP);
      std::copy(m + src, m + src + kP, out_m + (size_t)o * kP);
      std::copy(v + src, v + src + kP, out_v + (size_t)o * kP);
      o += 1;
      continue;
    }
    if (!(f & 4)) {
      for (int c = 0; c < 2; ++c) {
        std::copy(P, P + kP, out_p + (size_t)(o + c) * kP);
        if (c == 0) {
          std::copy(m + src, m + src + kP, out_m + (size_t)o * kP);
          std::copy(v + src, v + src + kP, out_v + (size_t)o * kP);
        } else {
          std::fill(out_m + (size_t)(o + 1) * kP, out_m + (size_t)(o + 2) * kP, 0.0f);
          std::fill(out_v + (size_t)(o + 1) * kP, out_v + (size_t)(o + 2) * kP, 0.0f);
        }
      }
    } else {
      for (uint32_t c = 0; c < 2; ++c) {
        float* Q = out_p + (size_t)(o + c) * kP;
        std::copy(P, P + kP, Q);
        float mean[3], ls[3];
        split_child(P, i, seed, c, mean, ls);
        for (int k = 0; k < 3; ++k) {
          Q[k] = mean[k];
          Q[3 + k] = ls[k];
        }
        std::fill(out_m + (size_t)(o + c) * kP, out_m + (size_t)(o + c + 1) * kP, 0.0f);
        std::fill(out_v + (size_t)(o + c) * kP, out_v + (size_t)(o + c + 1) * kP, 0.0f);
      }
    }
    o += 2;
  }
  if (counts4) {
    counts4[0] = n;
    counts4[1] = o;
    counts4[2] = std::min(cands, budget);
    counts4[3] = n - kept;
  }
  return 0;
}

// FP64 loss (no freezing) — for sanity checks.
double orc_gs_loss_f64(const float* params, uint32_t n, int deg, const float* views, uint32_t nv, uint32_t W,
                       uint32_t H, const float* bg, const float* tgt_all, const uint32_t* tids, double lambda,
                       int kind) {
  std::vector<double> p((size_t)n * kP);
  for (size_t i = 0; i < p.size(); ++i) p[i] = params[i];
  return total_loss<double>(p.data(), n, deg, views, nv, W, H, bg, tgt_all, tids, lambda, kind, nullptr, false);
}

// FP64 central differences of the loss w.r.t. the flat parameter indices
// pidx[0..np) (index = gaussian * 64 + field), step h = h_rel * max(|p|, 1e-3),
// with the base point's discrete decisions frozen.
int orc_gs_loss_cd(const float* params, uint32_t n, int deg, const float* views, uint32_t nv, uint32_t W, uint32_t H,
                   const float* bg, const float* tgt_all, const uint32_t* tids, double lambda, int kind,
                   const uint32_t* pidx, uint32_t npidx, double h_rel, double* out) {
  std::vector<double> p((size_t)n * kP);
  for (size_t i = 0; i < p.size(); ++i) p[i] = params[i];
  Frozen frz;
  total_loss<double>(p.data(), n, deg, views, nv, W, H, bg, tgt_all, tids, lambda, kind, &frz, false);
#pragma omp parallel for schedule(dynamic, 1)
  for (long k = 0; k < (long)npidx; ++k) {
    std::vector<double> q(p);
    const size_t j = pidx[k];
    const double h = h_rel * std::max(std::fabs(p[j]), 1e-3);
    q[j] = p[j] + h;
    const double lp =
        total_loss<double>(q.data(), n, deg, views, nv, W, H, bg, tgt_all, tids, lambda, kind, &frz, true);
    q[j] = p[j] - h;
    const double lm =
        total_loss<double>(q.data(), n, deg, views, nv, W, H, bg, tgt_all, tids, lambda, kind, &frz, true);
    out[k] = (lp - lm) / (2 * h);
  }
  return 0;
}

}  // extern "C"
