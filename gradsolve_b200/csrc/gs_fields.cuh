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
  FIELD_LINEAR = 4,  // the ABI passes FIELD_LINEAR * 1000 + D
  FIELD_ROBERTSON = 10,
  FIELD_LORENZ3 = 11,
};

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
