// gs_fields.cuh -- the registered right-hand sides, their hand-written VJPs and (for the
// stiff path) analytic Jacobians.
//
// Every RHS is written in the reference's textual operation order so the float64 kernel
// tracks the reference to rounding level:
//   Lorenz     gradsolve/warp/_warp_kernel.py:111-130 (sigma = 10, beta = 8/3, p = [rho])
//   Lorenz3    the same RHS with p = [sigma, beta, rho] read from the parameters (the
//              reference's 3-column "lorenz" problem, gradsolve/warp/warp_ode.py:575-588)
//   VdP        gradsolve/warp/_warp_kernel.py:158-174 (p = [mu])
//   Linear<D>  gradsolve/warp/_warp_kernel.py:133-155 (dy = 1.01 y, p ignored)
//   LotkaVolterra  dx = a x - b x y, dy = d x y - g y, p = [a, b, g, d]; the reference has
//              no built-in LV field (it is reachable only through register_jax_field,
//              gradsolve/warp/jax_field.py:393-447), so this is the hand-written
//              counterpart of that generated field.
//   Robertson  gradsolve/warp/_warp_rosenbrock.py:96-139 (p = [k1, k2, k3]); the analytic
//              Jacobian is the one of _warp_rosenbrock.py:121-137.
//   Lorenz96<D> gradsolve/warp/_warp_kernel.py:175-195: dy_i = (y_{i+1} - y_{i-2}) y_{i-1}
//              - y_i + F, cyclic indices, p = [F], D >= 4 (the reference's lorenz96_<D>)
//   Hires      gradsolve/warp/_warp_rosenbrock.py:142-216: HIRES-8 (Hairer & Wanner IV.10),
//              autonomous, p ignored; analytic Jacobian as in :186-214.
//
// Fields that can be integrated by a group of lanes (D > 8: Linear<D>, Lorenz96<D>) also
// give their right-hand side and VJP on a contiguous block of components, with the few
// neighbouring components they read (a cyclic stencil) passed in beside the block:
//   RHS_LO, RHS_HI                 components below / above the block rhs_block reads
//   rhs_block<C>(yb, p, dy)        yb[RHS_LO + k] = y_{i0+k}, k in [-RHS_LO, C + RHS_HI);
//                                  dy[k] = f_{i0+k}(y, p), k < C
//   VJP_YLO, VJP_YHI, VJP_WLO, VJP_WHI, and
//   vjp_block<C>(yb, wb, p, gy, gp) gy[k] += ((df/dy)^T w)_{i0+k}; gp += the block's share of
//                                  (df/dp)^T w (the shares of all blocks sum to it)
//
// Contract of each field F (R = double or float):
//   rhs(y, p, dy)                 dy = f(y, p)           (all fields are autonomous)
//   rhs_delta(y, p, d, df)        df = f(y + d, p) - f(y, p), expanded so that no large
//                                 terms cancel (used by the float32-stage kernels, where y
//                                 is the float64 state rounded to float and d is small)
//   vjp(y, p, w, gy, gp)          gy += (df/dy)^T w, gp += (df/dp)^T w
//   jac(y, p, J)                  J = df/dy, row-major D x D          (stiff fields)
//   jac_contract_grad(y,p,G,gy,gp) gy += d/dy <G, J(y,p)>, gp += d/dp <G, J(y,p)>
#pragma once

namespace gs {

#define GS_HD __host__ __device__ __forceinline__

enum FieldId : int {
  FIELD_LORENZ = 1,
  FIELD_VDP = 2,
  FIELD_LOTKA_VOLTERRA = 3,
  FIELD_LINEAR = 4,     // the ABI passes FIELD_LINEAR * 1000 + D
  FIELD_LORENZ96 = 5,   // the ABI passes FIELD_LORENZ96 * 1000 + D
  FIELD_ROBERTSON = 10,
  FIELD_LORENZ3 = 11,
  FIELD_HIRES = 12,
};

// Largest state dimension of the fused lanes (the reference refuses larger ones before
// launch on the GPU: _GPU_VEC_DIM_CEILING, gradsolve/warp/warp_ode.py:75-81).
constexpr int kMaxDim = 64;

// Lanes that share one trajectory for a field of dimension D: 1 up to D = 8; above, the
// smallest power of two G with D = G*C and C <= 4 components per lane, else the largest one
// with C >= 2 (a stencil reaches two components into the neighbouring lane's block), else 1
// (odd D: one thread per trajectory).
constexpr int coop_group(int D) {
  if (D <= 8) return 1;
  int best = 1;
  for (int g = 2; g <= 32; g *= 2) {
    if (D % g == 0 && D / g >= 2) {
      best = g;
      if (D / g <= 4) return g;
    }
  }
  return best;
}

struct Lorenz {
  static constexpr int D = 3, P = 1;
  template <class R>
  static GS_HD void rhs(const R* y, const R* p, R* dy) {
    const R sigma = R(10.0);
    const R beta = R(8.0) / R(3.0);
    const R rho = p[0];
    dy[0] = sigma * (y[1] - y[0]);
    dy[1] = rho * y[0] - y[1] - y[0] * y[2];
    dy[2] = y[0] * y[1] - beta * y[2];
  }
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R* p, const R* d, R* df) {
    const R sigma = R(10.0);
    const R beta = R(8.0) / R(3.0);
    const R rho = p[0];
    df[0] = sigma * (d[1] - d[0]);
    df[1] = rho * d[0] - d[1] - (y[0] * d[2] + d[0] * (y[2] + d[2]));
    df[2] = y[0] * d[1] + d[0] * (y[1] + d[1]) - beta * d[2];
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {
    const R sigma = R(10.0);
    const R beta = R(8.0) / R(3.0);
    const R rho = p[0];
    gy[0] += -sigma * w[0] + (rho - y[2]) * w[1] + y[1] * w[2];
    gy[1] += sigma * w[0] - w[1] + y[0] * w[2];
    gy[2] += -y[0] * w[1] - beta * w[2];
    gp[0] += y[0] * w[1];
  }
};

struct Lorenz3 {
  static constexpr int D = 3, P = 3;
  template <class R>
  static GS_HD void rhs(const R* y, const R* p, R* dy) {
    const R sigma = p[0], beta = p[1], rho = p[2];
    dy[0] = sigma * (y[1] - y[0]);
    dy[1] = rho * y[0] - y[1] - y[0] * y[2];
    dy[2] = y[0] * y[1] - beta * y[2];
  }
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R* p, const R* d, R* df) {
    const R sigma = p[0], beta = p[1], rho = p[2];
    df[0] = sigma * (d[1] - d[0]);
    df[1] = rho * d[0] - d[1] - (y[0] * d[2] + d[0] * (y[2] + d[2]));
    df[2] = y[0] * d[1] + d[0] * (y[1] + d[1]) - beta * d[2];
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {
    const R sigma = p[0], beta = p[1], rho = p[2];
    gy[0] += -sigma * w[0] + (rho - y[2]) * w[1] + y[1] * w[2];
    gy[1] += sigma * w[0] - w[1] + y[0] * w[2];
    gy[2] += -y[0] * w[1] - beta * w[2];
    gp[0] += (y[1] - y[0]) * w[0];
    gp[1] += -y[2] * w[2];
    gp[2] += y[0] * w[1];
  }
};

struct VdP {
  static constexpr int D = 2, P = 1;
  template <class R>
  static GS_HD void rhs(const R* y, const R* p, R* dy) {
    const R x = y[0], v = y[1], mu = p[0];
    dy[0] = v;
    dy[1] = mu * ((R(1.0) - x * x) * v - x);
  }
  // f1(x+dx, v+dv) - f1(x, v) = mu [ (1 - x^2) dv - (2x + dx) dx (v + dv) - dx ]
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R* p, const R* d, R* df) {
    const R x = y[0], v = y[1], mu = p[0], dx = d[0], dv = d[1];
    df[0] = dv;
    df[1] = mu * ((R(1.0) - x * x) * dv - (R(2.0) * x + dx) * dx * (v + dv) - dx);
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {
    const R x = y[0], v = y[1], mu = p[0];
    gy[0] += w[1] * mu * (R(-2.0) * x * v - R(1.0));
    gy[1] += w[0] + w[1] * mu * (R(1.0) - x * x);
    gp[0] += w[1] * ((R(1.0) - x * x) * v - x);
  }
  // J = [[0, 1], [mu (-2 x v - 1), mu (1 - x^2)]]  (for Rosenbrock23 at large mu)
  template <class R>
  static GS_HD void jac(const R* y, const R* p, R* J) {
    const R x = y[0], v = y[1], mu = p[0];
    J[0] = R(0.0);
    J[1] = R(1.0);
    J[2] = mu * (R(-2.0) * x * v - R(1.0));
    J[3] = mu * (R(1.0) - x * x);
  }
  template <class R>
  static GS_HD void jac_contract_grad(const R* y, const R* p, const R* G, R* gy, R* gp) {
    const R x = y[0], v = y[1], mu = p[0];
    gy[0] += R(-2.0) * mu * (G[2] * v + G[3] * x);
    gy[1] += R(-2.0) * mu * x * G[2];
    gp[0] += G[2] * (R(-2.0) * x * v - R(1.0)) + G[3] * (R(1.0) - x * x);
  }
};

struct LotkaVolterra {
  static constexpr int D = 2, P = 4;
  template <class R>
  static GS_HD void rhs(const R* y, const R* p, R* dy) {
    const R x = y[0], u = y[1];
    dy[0] = p[0] * x - p[1] * x * u;
    dy[1] = p[3] * x * u - p[2] * u;
  }
  // (x+dx)(u+du) - x u = x du + dx (u + du)
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R* p, const R* d, R* df) {
    const R dxu = y[0] * d[1] + d[0] * (y[1] + d[1]);
    df[0] = p[0] * d[0] - p[1] * dxu;
    df[1] = p[3] * dxu - p[2] * d[1];
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {
    const R x = y[0], u = y[1];
    gy[0] += (p[0] - p[1] * u) * w[0] + p[3] * u * w[1];
    gy[1] += -p[1] * x * w[0] + (p[3] * x - p[2]) * w[1];
    gp[0] += x * w[0];
    gp[1] += -x * u * w[0];
    gp[2] += -u * w[1];
    gp[3] += x * u * w[1];
  }
};

template <int DD>
struct Linear {
  static constexpr int D = DD, P = 1;
  static constexpr int GROUP = coop_group(DD);
  static constexpr int RHS_LO = 0, RHS_HI = 0, VJP_YLO = 0, VJP_YHI = 0, VJP_WLO = 0,
                       VJP_WHI = 0;
  template <int C, class R>
  static GS_HD void rhs_block(const R* yb, const R*, R* dy) {
#pragma unroll
    for (int k = 0; k < C; ++k) dy[k] = R(1.01) * yb[k];
  }
  template <int C, class R>
  static GS_HD void vjp_block(const R*, const R* wb, const R*, R* gy, R*) {
#pragma unroll
    for (int k = 0; k < C; ++k) gy[k] += R(1.01) * wb[k];
  }
  template <class R>
  static GS_HD void rhs(const R* y, const R*, R* dy) {
#pragma unroll
    for (int i = 0; i < D; ++i) dy[i] = R(1.01) * y[i];
  }
  template <class R>
  static GS_HD void rhs_delta(const R*, const R*, const R* d, R* df) {
#pragma unroll
    for (int i = 0; i < D; ++i) df[i] = R(1.01) * d[i];
  }
  template <class R>
  static GS_HD void vjp(const R*, const R*, const R* w, R* gy, R*) {
#pragma unroll
    for (int i = 0; i < D; ++i) gy[i] += R(1.01) * w[i];
  }
  template <class R>
  static GS_HD void jac(const R*, const R*, R* J) {
#pragma unroll
    for (int a = 0; a < D * D; ++a) J[a] = R(0.0);
#pragma unroll
    for (int i = 0; i < D; ++i) J[i * D + i] = R(1.01);
  }
  template <class R>
  static GS_HD void jac_contract_grad(const R*, const R*, const R*, R*, R*) {}
};

template <int DD>
struct Lorenz96 {
  static_assert(DD >= 4, "lorenz96 needs D >= 4 (four distinct stencil components)");
  static constexpr int D = DD, P = 1;
  static constexpr int GROUP = coop_group(DD);
  static constexpr int RHS_LO = 2, RHS_HI = 1, VJP_YLO = 2, VJP_YHI = 2, VJP_WLO = 1,
                       VJP_WHI = 2;
  // (y_{i+1} - y_{i-2}) * y_{i-1} - y_i + F, the reference's operation order
  template <int C, class R>
  static GS_HD void rhs_block(const R* yb, const R* p, R* dy) {
#pragma unroll
    for (int k = 0; k < C; ++k) dy[k] = (yb[k + 3] - yb[k]) * yb[k + 1] - yb[k + 2] + p[0];
  }
  // ((df/dy)^T w)_j = w_{j-1} y_{j-2} - w_{j+2} y_{j+1} + w_{j+1} (y_{j+2} - y_{j-1}) - w_j;
  // d f_i / dF = 1
  template <int C, class R>
  static GS_HD void vjp_block(const R* yb, const R* wb, const R*, R* gy, R* gp) {
#pragma unroll
    for (int k = 0; k < C; ++k) {
      const R* y = yb + k + 2;  // y[d] = y_{j+d}
      const R* w = wb + k + 1;  // w[d] = w_{j+d}
      gy[k] += w[-1] * y[-2] - w[2] * y[1] + w[1] * (y[2] - y[-1]) - w[0];
      gp[0] += w[0];
    }
  }
  template <class R>
  static GS_HD void rhs(const R* y, const R* p, R* dy) {
#pragma unroll
    for (int i = 0; i < D; ++i)
      dy[i] = (y[(i + 1) % D] - y[(i + D - 2) % D]) * y[(i + D - 1) % D] - y[i] + p[0];
  }
  // f(y + d) - f(y) = (d_{i+1} - d_{i-2}) (y_{i-1} + d_{i-1}) + (y_{i+1} - y_{i-2}) d_{i-1} - d_i
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R*, const R* d, R* df) {
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const int a = (i + 1) % D, b = (i + D - 2) % D, c = (i + D - 1) % D;
      df[i] = (d[a] - d[b]) * (y[c] + d[c]) + (y[a] - y[b]) * d[c] - d[i];
    }
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R*, const R* w, R* gy, R* gp) {
#pragma unroll
    for (int j = 0; j < D; ++j) {
      const int m1 = (j + D - 1) % D, m2 = (j + D - 2) % D, p1 = (j + 1) % D, p2 = (j + 2) % D;
      gy[j] += w[m1] * y[m2] - w[p2] * y[p1] + w[p1] * (y[p2] - y[m1]) - w[j];
      gp[0] += w[j];
    }
  }
};

struct Hires {
  static constexpr int D = 8, P = 1;  // p is a placeholder: HIRES has no free parameters
  template <class R>
  static GS_HD void rhs(const R* y, const R*, R* dy) {
    dy[0] = R(-1.71) * y[0] + R(0.43) * y[1] + R(8.32) * y[2] + R(0.0007);
    dy[1] = R(1.71) * y[0] - R(8.75) * y[1];
    dy[2] = R(-10.03) * y[2] + R(0.43) * y[3] + R(0.035) * y[4];
    dy[3] = R(8.32) * y[1] + R(1.71) * y[2] - R(1.12) * y[3];
    dy[4] = R(-1.745) * y[4] + R(0.43) * y[5] + R(0.43) * y[6];
    dy[5] = R(-280.0) * y[5] * y[7] + R(0.69) * y[3] + R(1.71) * y[4] - R(0.43) * y[5] +
            R(0.69) * y[6];
    dy[6] = R(280.0) * y[5] * y[7] - R(1.81) * y[6];
    dy[7] = R(-280.0) * y[5] * y[7] + R(1.81) * y[6];
  }
  // linear terms in d, and (y5 + d5)(y7 + d7) - y5 y7 = y5 d7 + d5 (y7 + d7)
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R*, const R* d, R* df) {
    const R q = y[5] * d[7] + d[5] * (y[7] + d[7]);
    df[0] = R(-1.71) * d[0] + R(0.43) * d[1] + R(8.32) * d[2];
    df[1] = R(1.71) * d[0] - R(8.75) * d[1];
    df[2] = R(-10.03) * d[2] + R(0.43) * d[3] + R(0.035) * d[4];
    df[3] = R(8.32) * d[1] + R(1.71) * d[2] - R(1.12) * d[3];
    df[4] = R(-1.745) * d[4] + R(0.43) * d[5] + R(0.43) * d[6];
    df[5] = R(-280.0) * q + R(0.69) * d[3] + R(1.71) * d[4] - R(0.43) * d[5] + R(0.69) * d[6];
    df[6] = R(280.0) * q - R(1.81) * d[6];
    df[7] = R(-280.0) * q + R(1.81) * d[6];
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R*, const R* w, R* gy, R*) {
    gy[0] += R(-1.71) * w[0] + R(1.71) * w[1];
    gy[1] += R(0.43) * w[0] - R(8.75) * w[1] + R(8.32) * w[3];
    gy[2] += R(8.32) * w[0] - R(10.03) * w[2] + R(1.71) * w[3];
    gy[3] += R(0.43) * w[2] - R(1.12) * w[3] + R(0.69) * w[5];
    gy[4] += R(0.035) * w[2] - R(1.745) * w[4] + R(1.71) * w[5];
    gy[5] += R(0.43) * w[4] + (R(-280.0) * y[7] - R(0.43)) * w[5] + R(280.0) * y[7] * w[6] -
             R(280.0) * y[7] * w[7];
    gy[6] += R(0.43) * w[4] + R(0.69) * w[5] - R(1.81) * w[6] + R(1.81) * w[7];
    gy[7] += R(-280.0) * y[5] * w[5] + R(280.0) * y[5] * w[6] - R(280.0) * y[5] * w[7];
  }
  template <class R>
  static GS_HD void jac(const R* y, const R*, R* J) {
#pragma unroll
    for (int a = 0; a < 64; ++a) J[a] = R(0.0);
    J[0 * 8 + 0] = R(-1.71); J[0 * 8 + 1] = R(0.43); J[0 * 8 + 2] = R(8.32);
    J[1 * 8 + 0] = R(1.71); J[1 * 8 + 1] = R(-8.75);
    J[2 * 8 + 2] = R(-10.03); J[2 * 8 + 3] = R(0.43); J[2 * 8 + 4] = R(0.035);
    J[3 * 8 + 1] = R(8.32); J[3 * 8 + 2] = R(1.71); J[3 * 8 + 3] = R(-1.12);
    J[4 * 8 + 4] = R(-1.745); J[4 * 8 + 5] = R(0.43); J[4 * 8 + 6] = R(0.43);
    J[5 * 8 + 3] = R(0.69); J[5 * 8 + 4] = R(1.71); J[5 * 8 + 5] = R(-280.0) * y[7] - R(0.43);
    J[5 * 8 + 6] = R(0.69); J[5 * 8 + 7] = R(-280.0) * y[5];
    J[6 * 8 + 5] = R(280.0) * y[7]; J[6 * 8 + 6] = R(-1.81); J[6 * 8 + 7] = R(280.0) * y[5];
    J[7 * 8 + 5] = R(-280.0) * y[7]; J[7 * 8 + 6] = R(1.81); J[7 * 8 + 7] = R(-280.0) * y[5];
  }
  // only J[5][5], J[6][5], J[7][5] (through y7) and J[5][7], J[6][7], J[7][7] (through y5)
  // depend on the state
  template <class R>
  static GS_HD void jac_contract_grad(const R*, const R*, const R* G, R* gy, R*) {
    gy[5] += R(-280.0) * G[5 * 8 + 7] + R(280.0) * G[6 * 8 + 7] - R(280.0) * G[7 * 8 + 7];
    gy[7] += R(-280.0) * G[5 * 8 + 5] + R(280.0) * G[6 * 8 + 5] - R(280.0) * G[7 * 8 + 5];
  }
};

// Group sizes built besides the default: half and twice it, where the lanes still hold equal
// blocks of 2 to 8 components (a stencil reaches two components into a neighbour's block;
// above 8 the lane's registers run out).
template <int D, int G>
constexpr bool group_built() {
  return G == coop_group(D) ||
         (G >= 2 && G <= 32 && coop_group(D) > 1 && (G == 2 * coop_group(D) ||
                                                      2 * G == coop_group(D)) &&
          D % G == 0 && D / G >= 2 && D / G <= 8);
}

// Lanes per trajectory of a field: its GROUP where it declares one (the stencil fields),
// else 1.
template <class F, class = void>
struct group_of {
  static constexpr int value = 1;
};
template <class F>
struct group_of<F, decltype(void(F::GROUP))> {
  static constexpr int value = F::GROUP;
};

struct Robertson {
  static constexpr int D = 3, P = 3;
  template <class R>
  static GS_HD void rhs(const R* y, const R* p, R* dy) {
    const R k1 = p[0], k2 = p[1], k3 = p[2];
    const R a = y[0], b = y[1], c = y[2];
    dy[0] = -k1 * a + k3 * b * c;
    dy[1] = k1 * a - k3 * b * c - k2 * b * b;
    dy[2] = k2 * b * b;
  }
  // with e = (b+db)(c+dc) - b c = b dc + db (c + dc) and q = (b+db)^2 - b^2 = db (2b + db)
  template <class R>
  static GS_HD void rhs_delta(const R* y, const R* p, const R* d, R* df) {
    const R k1 = p[0], k2 = p[1], k3 = p[2];
    const R e = y[1] * d[2] + d[1] * (y[2] + d[2]);
    const R q = d[1] * (R(2.0) * y[1] + d[1]);
    df[0] = -k1 * d[0] + k3 * e;
    df[1] = k1 * d[0] - k3 * e - k2 * q;
    df[2] = k2 * q;
  }
  template <class R>
  static GS_HD void vjp(const R* y, const R* p, const R* w, R* gy, R* gp) {
    const R k1 = p[0], k2 = p[1], k3 = p[2];
    const R a = y[0], b = y[1], c = y[2];
    gy[0] += -k1 * w[0] + k1 * w[1];
    gy[1] += k3 * c * w[0] + (-k3 * c - R(2.0) * k2 * b) * w[1] + R(2.0) * k2 * b * w[2];
    gy[2] += k3 * b * w[0] - k3 * b * w[1];
    gp[0] += -a * w[0] + a * w[1];
    gp[1] += -b * b * w[1] + b * b * w[2];
    gp[2] += b * c * w[0] - b * c * w[1];
  }
  template <class R>
  static GS_HD void jac(const R* y, const R* p, R* J) {
    const R k1 = p[0], k2 = p[1], k3 = p[2], b = y[1], c = y[2];
    J[0] = -k1;
    J[1] = k3 * c;
    J[2] = k3 * b;
    J[3] = k1;
    J[4] = -k3 * c - R(2.0) * k2 * b;
    J[5] = -k3 * b;
    J[6] = R(0.0);
    J[7] = R(2.0) * k2 * b;
    J[8] = R(0.0);
  }
  template <class R>
  static GS_HD void jac_contract_grad(const R* y, const R* p, const R* G, R* gy, R* gp) {
    const R k2 = p[1], k3 = p[2], b = y[1], c = y[2];
    gy[1] += k3 * G[2] - R(2.0) * k2 * G[4] - k3 * G[5] + R(2.0) * k2 * G[7];
    gy[2] += k3 * G[1] - k3 * G[4];
    gp[0] += -G[0] + G[3];
    gp[1] += R(-2.0) * b * G[4] + R(2.0) * b * G[7];
    gp[2] += c * G[1] + b * G[2] - c * G[4] - b * G[5];
  }
};

}  // namespace gs
