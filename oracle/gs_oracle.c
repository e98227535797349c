/*
 * gs_oracle.c -- CPU oracle for the ensemble adaptive solve and its replay adjoint.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the reference result that the CUDA path is
 * compared against; it is never linked into, loaded by, or called from the product library
 * (gradsolve_b200/, libgsolve.so).  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load it.
 *
 * What it restates (plain C, evaluated in the reference's own operation order,
 * compiled with -ffp-contract=off so no multiply-add is fused):
 *
 *   tsit5 record   gradsolve/solvers/tsit5_replay.py:62-124 (tsit5_adaptive) -- FSAL,
 *                  WRMS error norm, I-controller run after accept AND reject, the last
 *                  step clamped with h = min(dt, t1 - t), max_steps counting attempts.
 *                  Tableau: gradsolve/solvers/tsit5_step.py:26-77.
 *                  numpy evaluates np.mean((e/sc)**2) sequentially for D < 8 and with
 *                  its 8-accumulator pairwise sum for D >= 8; wrms_sum() follows that.
 *   tsit5 replay   gradsolve/warp/warp_replay.py:30-55 (replay_solve_jax) over
 *                  gradsolve/solvers/tsit5_step.py:80-102 (tsit5_step, k7 computed and
 *                  the B7*k7 term kept); dt == 0 is an identity step.
 *   tsit5 vjp      reverse-mode derivative of that replay w.r.t. y0 and params with the
 *                  dts held fixed (the frozen-controller adjoint that jax.grad computes
 *                  through warp_replay.py:30-55).  Hand-derived; all states stored.
 *   ros23 record   gradsolve/warp/_warp_rosenbrock.py:383-452 (the fused kernel's
 *                  arithmetic: W = I - d*h*J, three partial-pivot Gaussian eliminations
 *                  with division, _gauss_solve :346-381) with the controller of
 *                  tests/_oracles/gradsolve_g2_spike_oracle.py:138-184 (exponent -1/3).
 *   ros23 replay   gradsolve/solvers/rosenbrock23_step.py:47-66 (no k3, J analytic).
 *   ros23 vjp      reverse-mode derivative of that replay, including the second-order
 *                  term d(J(y,p)^T-contraction)/d(y,p) through W.
 *
 * Fields (RHS in the reference's textual operation order):
 *   lorenz   gradsolve/warp/_warp_kernel.py:111-130, sigma=10, beta=8/3, p=[rho]
 *   lorenz3  the same RHS with p=[sigma, beta, rho]
 *   vdp      gradsolve/warp/_warp_kernel.py:158-174, p=[mu]
 *   lv       Lotka-Volterra dx = a*x - b*x*y, dy = d*x*y - g*y, p=[a,b,g,d]
 *            (absent from the reference's registry; reachable there only through
 *            register_jax_field, gradsolve/warp/jax_field.py:393-447)
 *   linear_D gradsolve/warp/_warp_kernel.py:133-155, dy = 1.01*y (p ignored)
 *   lorenz96_D gradsolve/warp/_warp_kernel.py:175-195, dy_i = (y_{i+1} - y_{i-2}) y_{i-1}
 *            - y_i + F, cyclic indices, p=[F], D >= 4
 *   robertson gradsolve/warp/_warp_rosenbrock.py:96-139, p=[k1,k2,k3]
 *   hires    gradsolve/warp/_warp_rosenbrock.py:142-216 (HIRES-8, autonomous, p ignored)
 *   linstiff gradsolve/warp/_warp_rosenbrock.py:219-252, f = A y with a constant D x D
 *            matrix A (set by gso_set_linstiff; p ignored)
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <pthread.h>
#include <stdatomic.h>

/* ---- Tsitouras (2011) tableau, the values of gradsolve/solvers/tsit5_step.py:31-77 ---- */
static const double C2 = 161.0 / 1000.0;
static const double C3 = 327.0 / 1000.0;
static const double C4 = 9.0 / 10.0;
static const double C5 = 0.9800255409045096857298102862870245954942137979563024768854764293221195950761080302604;
static const double C6 = 1.0;
static const double A21 = 161.0 / 1000.0;
static const double A31 = -0.8480655492356988544426874250230774675121177393430391537369234245294192976164141156943e-2;
static const double A32 = 0.3354806554923569885444268742502307746751211773934303915373692342452941929761641411569;
static const double A41 = 2.897153057105493432130432594192938764924887287701866490314866693455023795137503079289;
static const double A42 = -6.359448489975074843148159912383825625952700647415626703305928850207288721235210244366;
static const double A43 = 4.362295432869581411017727318190886861027813359713760212991062156752264926097707165077;
static const double A51 = 5.325864828439256604428877920840511317836476253097040101202360397727981648835607691791;
static const double A52 = -11.74888356406282787774717033978577296188744178259862899288666928009020615663593781589;
static const double A53 = 7.495539342889836208304604784564358155658679161518186721010132816213648793440552049753;
static const double A54 = -0.9249506636175524925650207933207191611349983406029535244034750452930469056411389539635e-1;
static const double A61 = 5.861455442946420028659251486982647890394337666164814434818157239052507339770711679748;
static const double A62 = -12.92096931784710929170611868178335939541780751955743459166312250439928519268343184452;
static const double A63 = 8.159367898576158643180400794539253485181918321135053305748355423955009222648673734986;
static const double A64 = -0.7158497328140099722453054252582973869127213147363544882721139659546372402303777878835e-1;
static const double A65 = -0.2826905039406838290900305721271224146717633626879770007617876201276764571291579142206e-1;
static const double B1 = 0.9646076681806522951816731316512876333711995238157997181903319145764851595234062815396e-1;
static const double B2 = 1.0 / 100.0;
static const double B3 = 0.4798896504144995747752495322905965199130404621990332488332634944254542060153074523509;
static const double B4 = 1.379008574103741893192274821856872770756462643091360525934940067397245698027561293331;
static const double B5 = -3.290069515436080679901047585711363850115683290894936158531296799594813811049925401677;
static const double B6 = 2.324710524099773982415355918398765796109060233222962411944060046314465391054716027841;
static const double B7 = 0.0;
/* e_i = b_i - bhat_i; the subtraction is evaluated in double exactly as the Python
 * module-level expressions are (tsit5_step.py:64-70). Filled by init_tableau(). */
static double E1, E2, E3, E4, E5, E6, E7;
static int tableau_ready = 0;

static void init_tableau(void) {
  if (tableau_ready) return;
  volatile double a, b;
  a = 0.9646076681806522951816731316512876333711995238157997181903319145764851595234062815396e-1;
  b = 0.9468075576583945807478876255758922856117527357724631226139574065785592789071067303271e-1;
  E1 = a - b;
  a = 1.0 / 100.0;
  b = 0.9183565540343253096776363936645313759813746240984095238905939532922955247253608687270e-2;
  E2 = a - b;
  a = 0.4798896504144995747752495322905965199130404621990332488332634944254542060153074523509;
  b = 0.4877705284247615707855642599631228241516691959761363774365216240304071651579571959813;
  E3 = a - b;
  a = 1.379008574103741893192274821856872770756462643091360525934940067397245698027561293331;
  b = 1.234297566930478985655109673884237654035539930748192848315425833500484878378061439761;
  E4 = a - b;
  a = -3.290069515436080679901047585711363850115683290894936158531296799594813811049925401677;
  b = 2.707712349983525454881109975059321670689605166938197378763992255714444407154902012702;
  E5 = a + b;
  a = 2.324710524099773982415355918398765796109060233222962411944060046314465391054716027841;
  b = 1.866628418170587035753719399566211498666255505244122593996591602841258328965767580089;
  E6 = a - b;
  a = -1.0;
  b = 66.0;
  E7 = a / b;
  tableau_ready = 1;
}

/* controller constants: tsit5_step.py:26 and _warp_rosenbrock.py:62-70 */
static const double SAFETY = 0.9, ERR_FLOOR = 1e-10, FAC_MIN = 0.2, FAC_MAX = 5.0;
static const double ORDER_EXP_TSIT5 = -0.2;

/* Rosenbrock23 coefficients: _warp_rosenbrock.py:62-63 (computed, not typed in). */
static double ROS_D, ROS_E32, ROS_EXP;

#define MAXD 64
#define MAXP 8

enum { F_LORENZ = 1, F_VDP = 2, F_LV = 3, F_LINEAR = 4, F_LORENZ96 = 5, F_ROBERTSON = 10,
       F_LORENZ3 = 11, F_HIRES = 12, F_LINSTIFF = 13 };

/* the constant matrix of the linstiff field (row-major, g_ls_D x g_ls_D) */
static double g_ls_A[MAXD * MAXD];
static int g_ls_D = 0;

int gso_set_linstiff(int D, const double* A) {
  if (D < 1 || D > MAXD) return -1;
  memcpy(g_ls_A, A, sizeof(double) * (size_t)D * (size_t)D);
  g_ls_D = D;
  return 0;
}

typedef struct {
  int id, D, P;
} field_t;

static int field_make(int code, field_t* f) {
  /* code = id * 1000 + D for linear, plain id otherwise */
  int id = code >= 1000 ? code / 1000 : code;
  int D = code >= 1000 ? code % 1000 : 0;
  f->id = id;
  switch (id) {
    case F_LORENZ: f->D = 3; f->P = 1; return 0;
    case F_VDP: f->D = 2; f->P = 1; return 0;
    case F_LV: f->D = 2; f->P = 4; return 0;
    case F_LINEAR: if (D < 1 || D > MAXD) return -1; f->D = D; f->P = 1; return 0;
    case F_LORENZ96: if (D < 4 || D > MAXD) return -1; f->D = D; f->P = 1; return 0;
    case F_ROBERTSON: f->D = 3; f->P = 3; return 0;
    case F_LORENZ3: f->D = 3; f->P = 3; return 0;
    case F_HIRES: f->D = 8; f->P = 1; return 0;
    case F_LINSTIFF: if (D < 1 || D != g_ls_D) return -1; f->D = D; f->P = 1; return 0;
  }
  return -1;
}

/* ---- right-hand sides, reference operation order ---- */
static void rhs(const field_t* f, const double* y, const double* p, double* dy) {
  switch (f->id) {
    case F_LORENZ: {
      const double sigma = 10.0, beta = 8.0 / 3.0, rho = p[0];
      dy[0] = sigma * (y[1] - y[0]);
      dy[1] = rho * y[0] - y[1] - y[0] * y[2];
      dy[2] = y[0] * y[1] - beta * y[2];
    } break;
    case F_LORENZ3: {
      const double sigma = p[0], beta = p[1], rho = p[2];
      dy[0] = sigma * (y[1] - y[0]);
      dy[1] = rho * y[0] - y[1] - y[0] * y[2];
      dy[2] = y[0] * y[1] - beta * y[2];
    } break;
    case F_VDP: {
      const double x = y[0], v = y[1], mu = p[0];
      dy[0] = v;
      dy[1] = mu * ((1.0 - x * x) * v - x);
    } break;
    case F_LV: {
      const double x = y[0], w = y[1];
      dy[0] = p[0] * x - p[1] * x * w;
      dy[1] = p[3] * x * w - p[2] * w;
    } break;
    case F_LINEAR:
      for (int i = 0; i < f->D; ++i) dy[i] = 1.01 * y[i];
      break;
    case F_LORENZ96: {
      const int D = f->D;
      for (int i = 0; i < D; ++i) {
        const int ip1 = (i + 1) % D, im1 = (i - 1 + D) % D, im2 = (i - 2 + D) % D;
        dy[i] = (y[ip1] - y[im2]) * y[im1] - y[i] + p[0];
      }
    } break;
    case F_ROBERTSON: {
      const double k1 = p[0], k2 = p[1], k3 = p[2];
      const double a = y[0], b = y[1], c = y[2];
      dy[0] = -k1 * a + k3 * b * c;
      dy[1] = k1 * a - k3 * b * c - k2 * b * b;
      dy[2] = k2 * b * b;
    } break;
    case F_HIRES:
      dy[0] = -1.71 * y[0] + 0.43 * y[1] + 8.32 * y[2] + 0.0007;
      dy[1] = 1.71 * y[0] - 8.75 * y[1];
      dy[2] = -10.03 * y[2] + 0.43 * y[3] + 0.035 * y[4];
      dy[3] = 8.32 * y[1] + 1.71 * y[2] - 1.12 * y[3];
      dy[4] = -1.745 * y[4] + 0.43 * y[5] + 0.43 * y[6];
      dy[5] = -280.0 * y[5] * y[7] + 0.69 * y[3] + 1.71 * y[4] - 0.43 * y[5] + 0.69 * y[6];
      dy[6] = 280.0 * y[5] * y[7] - 1.81 * y[6];
      dy[7] = -280.0 * y[5] * y[7] + 1.81 * y[6];
      break;
    case F_LINSTIFF: {
      const int D = f->D;
      for (int i = 0; i < D; ++i) {
        double acc = 0.0;
        for (int k = 0; k < D; ++k) acc += g_ls_A[i * D + k] * y[k];
        dy[i] = acc;
      }
    } break;
  }
}

/* Accumulate  gy += (df/dy)^T w  and  gp += (df/dp)^T w  at (y, p). */
static void rhs_vjp(const field_t* f, const double* y, const double* p, const double* w,
                    double* gy, double* gp) {
  switch (f->id) {
    case F_LORENZ: {
      const double sigma = 10.0, beta = 8.0 / 3.0, rho = p[0];
      gy[0] += -sigma * w[0] + (rho - y[2]) * w[1] + y[1] * w[2];
      gy[1] += sigma * w[0] - w[1] + y[0] * w[2];
      gy[2] += -y[0] * w[1] - beta * w[2];
      gp[0] += y[0] * w[1];
    } break;
    case F_LORENZ3: {
      const double sigma = p[0], beta = p[1], rho = p[2];
      gy[0] += -sigma * w[0] + (rho - y[2]) * w[1] + y[1] * w[2];
      gy[1] += sigma * w[0] - w[1] + y[0] * w[2];
      gy[2] += -y[0] * w[1] - beta * w[2];
      gp[0] += (y[1] - y[0]) * w[0];
      gp[1] += -y[2] * w[2];
      gp[2] += y[0] * w[1];
    } break;
    case F_VDP: {
      const double x = y[0], v = y[1], mu = p[0];
      gy[0] += w[1] * mu * (-2.0 * x * v - 1.0);
      gy[1] += w[0] + w[1] * mu * (1.0 - x * x);
      gp[0] += w[1] * ((1.0 - x * x) * v - x);
    } break;
    case F_LV: {
      const double x = y[0], u = y[1];
      gy[0] += (p[0] - p[1] * u) * w[0] + p[3] * u * w[1];
      gy[1] += -p[1] * x * w[0] + (p[3] * x - p[2]) * w[1];
      gp[0] += x * w[0];
      gp[1] += -x * u * w[0];
      gp[2] += -u * w[1];
      gp[3] += x * u * w[1];
    } break;
    case F_LINEAR:
      for (int i = 0; i < f->D; ++i) gy[i] += 1.01 * w[i];
      break;
    case F_LORENZ96: {
      const int D = f->D;
      for (int i = 0; i < D; ++i) {
        const int ip1 = (i + 1) % D, im1 = (i - 1 + D) % D, im2 = (i - 2 + D) % D;
        gy[ip1] += y[im1] * w[i];
        gy[im2] += -y[im1] * w[i];
        gy[im1] += (y[ip1] - y[im2]) * w[i];
        gy[i] += -w[i];
        gp[0] += w[i];
      }
    } break;
    case F_HIRES:
      gy[0] += -1.71 * w[0] + 1.71 * w[1];
      gy[1] += 0.43 * w[0] - 8.75 * w[1] + 8.32 * w[3];
      gy[2] += 8.32 * w[0] - 10.03 * w[2] + 1.71 * w[3];
      gy[3] += 0.43 * w[2] - 1.12 * w[3] + 0.69 * w[5];
      gy[4] += 0.035 * w[2] - 1.745 * w[4] + 1.71 * w[5];
      gy[5] += 0.43 * w[4] + (-280.0 * y[7] - 0.43) * w[5] + 280.0 * y[7] * w[6] -
               280.0 * y[7] * w[7];
      gy[6] += 0.43 * w[4] + 0.69 * w[5] - 1.81 * w[6] + 1.81 * w[7];
      gy[7] += -280.0 * y[5] * w[5] + 280.0 * y[5] * w[6] - 280.0 * y[5] * w[7];
      break;
    case F_LINSTIFF: {
      const int D = f->D;
      for (int k = 0; k < D; ++k) {
        double acc = 0.0;
        for (int i = 0; i < D; ++i) acc += g_ls_A[i * D + k] * w[i];
        gy[k] += acc;
      }
    } break;
    case F_ROBERTSON: {
      const double k1 = p[0], k2 = p[1], k3 = p[2];
      const double a = y[0], b = y[1], c = y[2];
      (void)a;
      gy[0] += -k1 * w[0] + k1 * w[1];
      gy[1] += k3 * c * w[0] + (-k3 * c - 2.0 * k2 * b) * w[1] + 2.0 * k2 * b * w[2];
      gy[2] += k3 * b * w[0] - k3 * b * w[1];
      gp[0] += -a * w[0] + a * w[1];
      gp[1] += -b * b * w[1] + b * b * w[2];
      gp[2] += b * c * w[0] - b * c * w[1];
    } break;
  }
}

/* Analytic Jacobian, row-major; _warp_rosenbrock.py:121-137 order. */
static void jac(const field_t* f, const double* y, const double* p, double* J) {
  const int D = f->D;
  memset(J, 0, sizeof(double) * D * D);
  switch (f->id) {
    case F_ROBERTSON: {
      const double k1 = p[0], k2 = p[1], k3 = p[2], b = y[1], c = y[2];
      J[0] = -k1;
      J[1] = k3 * c;
      J[2] = k3 * b;
      J[3] = k1;
      J[4] = -k3 * c - 2.0 * k2 * b;
      J[5] = -k3 * b;
      J[6] = 0.0;
      J[7] = 2.0 * k2 * b;
      J[8] = 0.0;
    } break;
    case F_LINEAR:
      for (int i = 0; i < D; ++i) J[i * D + i] = 1.01;
      break;
    case F_HIRES:
      J[0 * 8 + 0] = -1.71; J[0 * 8 + 1] = 0.43; J[0 * 8 + 2] = 8.32;
      J[1 * 8 + 0] = 1.71; J[1 * 8 + 1] = -8.75;
      J[2 * 8 + 2] = -10.03; J[2 * 8 + 3] = 0.43; J[2 * 8 + 4] = 0.035;
      J[3 * 8 + 1] = 8.32; J[3 * 8 + 2] = 1.71; J[3 * 8 + 3] = -1.12;
      J[4 * 8 + 4] = -1.745; J[4 * 8 + 5] = 0.43; J[4 * 8 + 6] = 0.43;
      J[5 * 8 + 3] = 0.69; J[5 * 8 + 4] = 1.71; J[5 * 8 + 5] = -280.0 * y[7] - 0.43;
      J[5 * 8 + 6] = 0.69; J[5 * 8 + 7] = -280.0 * y[5];
      J[6 * 8 + 5] = 280.0 * y[7]; J[6 * 8 + 6] = -1.81; J[6 * 8 + 7] = 280.0 * y[5];
      J[7 * 8 + 5] = -280.0 * y[7]; J[7 * 8 + 6] = 1.81; J[7 * 8 + 7] = -280.0 * y[5];
      break;
    case F_LINSTIFF:
      memcpy(J, g_ls_A, sizeof(double) * (size_t)D * (size_t)D);
      break;
    default: {
      /* generic: J^T e_j columns through the VJP (used only by the stiff path on a
       * non-stiff field, which the tests do for cross-checks) */
      double w[MAXD], gy[MAXD], gp[MAXP];
      for (int r = 0; r < D; ++r) {
        for (int i = 0; i < D; ++i) { w[i] = (i == r) ? 1.0 : 0.0; gy[i] = 0.0; }
        for (int k = 0; k < MAXP; ++k) gp[k] = 0.0;
        rhs_vjp(f, y, p, w, gy, gp);
        for (int cc = 0; cc < D; ++cc) J[r * D + cc] = gy[cc];
      }
    }
  }
}

/* Accumulate the contraction derivative: for a fixed DxD matrix G,
 * gy += d/dy sum_ab G_ab J_ab(y,p),  gp += d/dp sum_ab G_ab J_ab(y,p). */
static void jac_contract_grad(const field_t* f, const double* y, const double* p,
                              const double* G, double* gy, double* gp) {
  switch (f->id) {
    case F_ROBERTSON: {
      const double k1 = p[0], k2 = p[1], k3 = p[2], b = y[1], c = y[2];
      (void)k1;
      gy[1] += k3 * G[2] - 2.0 * k2 * G[4] - k3 * G[5] + 2.0 * k2 * G[7];
      gy[2] += k3 * G[1] - k3 * G[4];
      gp[0] += -G[0] + G[3];
      gp[1] += -2.0 * b * G[4] + 2.0 * b * G[7];
      gp[2] += c * G[1] + b * G[2] - c * G[4] - b * G[5];
    } break;
    case F_VDP: {
      const double x = y[0], v = y[1], mu = p[0];
      gy[0] += -2.0 * mu * (G[2] * v + G[3] * x);
      gy[1] += -2.0 * mu * x * G[2];
      gp[0] += G[2] * (-2.0 * x * v - 1.0) + G[3] * (1.0 - x * x);
    } break;
    case F_HIRES:
      gy[5] += -280.0 * G[5 * 8 + 7] + 280.0 * G[6 * 8 + 7] - 280.0 * G[7 * 8 + 7];
      gy[7] += -280.0 * G[5 * 8 + 5] + 280.0 * G[6 * 8 + 5] - 280.0 * G[7 * 8 + 5];
      break;
    default: break; /* constant Jacobian (linear, linstiff) */
  }
}

/* numpy's add.reduce order: sequential below 8 terms, 8-way pairwise from 8 to 128. */
static double wrms_sum(const double* a, int n) {
  if (n < 8) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += a[i];
    return s;
  }
  double r[8];
  for (int j = 0; j < 8; ++j) r[j] = a[j];
  int i = 8;
  for (; i < n - (n % 8); i += 8)
    for (int j = 0; j < 8; ++j) r[j] += a[i + j];
  double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
  for (; i < n; ++i) res += a[i];
  return res;
}

static double wrms(const double* e, const double* y, const double* ynew, double rtol,
                   double atol, int D) {
  double q[MAXD];
  for (int i = 0; i < D; ++i) {
    double ay = fabs(y[i]), an = fabs(ynew[i]);
    double sc = atol + rtol * (ay >= an ? ay : an);
    double c = e[i] / sc;
    q[i] = c * c;
  }
  return sqrt(wrms_sum(q, D) / (double)D);
}

static double controller(double err, double h, double order_exp) {
  double e = err > ERR_FLOOR ? err : ERR_FLOOR;
  if (err != err) e = err;
  double fac = SAFETY * pow(e, order_exp);
  double lo = fac > FAC_MIN ? fac : FAC_MIN;
  if (fac != fac) lo = fac;
  double c = FAC_MAX < lo ? FAC_MAX : lo;
  return h * c;
}

/* ---------------------------------------------------------------------------------- */
/* Tsit5                                                                              */
/* ---------------------------------------------------------------------------------- */

/* One trajectory of tsit5_adaptive (tsit5_replay.py:62-124). dts gets the accepted h's
 * (up to cap entries). Returns status: 0 reached t1, 1 max_steps exhausted, 3 cap full. */
static int tsit5_one(const field_t* f, const double* y0, const double* p, double t0,
                     double t1, double rtol, double atol, double dt0, int max_steps,
                     int cap, double* dts, double* yf, int* n_acc, int* n_rej) {
  const int D = f->D;
  double y[MAXD], k1[MAXD], k2[MAXD], k3[MAXD], k4[MAXD], k5[MAXD], k6[MAXD], k7[MAXD];
  double s[MAXD], y5[MAXD], e[MAXD];
  for (int i = 0; i < D; ++i) y[i] = y0[i];
  double t = t0, dt = dt0;
  rhs(f, y, p, k1);
  int acc = 0, rej = 0, status = 0;
  for (int it = 0; it < max_steps; ++it) {
    if (t >= t1) break;
    double h = (t1 - t < dt) ? (t1 - t) : dt;
    for (int i = 0; i < D; ++i) s[i] = y[i] + h * (A21 * k1[i]);
    rhs(f, s, p, k2);
    for (int i = 0; i < D; ++i) s[i] = y[i] + h * (A31 * k1[i] + A32 * k2[i]);
    rhs(f, s, p, k3);
    for (int i = 0; i < D; ++i) s[i] = y[i] + h * (A41 * k1[i] + A42 * k2[i] + A43 * k3[i]);
    rhs(f, s, p, k4);
    for (int i = 0; i < D; ++i)
      s[i] = y[i] + h * (A51 * k1[i] + A52 * k2[i] + A53 * k3[i] + A54 * k4[i]);
    rhs(f, s, p, k5);
    for (int i = 0; i < D; ++i)
      s[i] = y[i] + h * (A61 * k1[i] + A62 * k2[i] + A63 * k3[i] + A64 * k4[i] + A65 * k5[i]);
    rhs(f, s, p, k6);
    for (int i = 0; i < D; ++i)
      y5[i] = y[i] + h * (B1 * k1[i] + B2 * k2[i] + B3 * k3[i] + B4 * k4[i] + B5 * k5[i] +
                          B6 * k6[i]);
    rhs(f, y5, p, k7);
    for (int i = 0; i < D; ++i)
      e[i] = h * (E1 * k1[i] + E2 * k2[i] + E3 * k3[i] + E4 * k4[i] + E5 * k5[i] +
                  E6 * k6[i] + E7 * k7[i]);
    double err = wrms(e, y, y5, rtol, atol, D);
    if (err <= 1.0) {
      if (acc >= cap) { status = 3; break; }
      t = t + h;
      for (int i = 0; i < D; ++i) { y[i] = y5[i]; k1[i] = k7[i]; }
      dts[acc] = h;
      ++acc;
    } else {
      ++rej;
    }
    dt = controller(err, h, ORDER_EXP_TSIT5);
  }
  if (status == 0 && !(t >= t1)) status = 1;
  for (int i = 0; i < D; ++i) yf[i] = y[i];
  *n_acc = acc;
  *n_rej = rej;
  return status;
}

/* tsit5_step (tsit5_step.py:80-102): stages s_1..s_7 and k_1..k_7, y_next. */
static void tsit5_stages(const field_t* f, const double* y, const double* p, double dt,
                         double S[7][MAXD], double K[7][MAXD], double* ynext) {
  const int D = f->D;
  for (int i = 0; i < D; ++i) S[0][i] = y[i];
  rhs(f, S[0], p, K[0]);
  for (int i = 0; i < D; ++i) S[1][i] = y[i] + dt * (A21 * K[0][i]);
  rhs(f, S[1], p, K[1]);
  for (int i = 0; i < D; ++i) S[2][i] = y[i] + dt * (A31 * K[0][i] + A32 * K[1][i]);
  rhs(f, S[2], p, K[2]);
  for (int i = 0; i < D; ++i)
    S[3][i] = y[i] + dt * (A41 * K[0][i] + A42 * K[1][i] + A43 * K[2][i]);
  rhs(f, S[3], p, K[3]);
  for (int i = 0; i < D; ++i)
    S[4][i] = y[i] + dt * (A51 * K[0][i] + A52 * K[1][i] + A53 * K[2][i] + A54 * K[3][i]);
  rhs(f, S[4], p, K[4]);
  for (int i = 0; i < D; ++i)
    S[5][i] = y[i] + dt * (A61 * K[0][i] + A62 * K[1][i] + A63 * K[2][i] + A64 * K[3][i] +
                           A65 * K[4][i]);
  rhs(f, S[5], p, K[5]);
  for (int i = 0; i < D; ++i)
    S[6][i] = y[i] + dt * (B1 * K[0][i] + B2 * K[1][i] + B3 * K[2][i] + B4 * K[3][i] +
                           B5 * K[4][i] + B6 * K[5][i]);
  rhs(f, S[6], p, K[6]);
  if (ynext)
    for (int i = 0; i < D; ++i)
      ynext[i] = y[i] + dt * (B1 * K[0][i] + B2 * K[1][i] + B3 * K[2][i] + B4 * K[3][i] +
                              B5 * K[4][i] + B6 * K[5][i] + B7 * K[6][i]);
}

/* Reverse of one tsit5_step at (y, dt): lam <- (dy'/dy)^T lam, gp += (dy'/dp)^T lam. */
static void tsit5_step_vjp(const field_t* f, const double* y, const double* p, double dt,
                           double* lam, double* gp) {
  const int D = f->D;
  double S[7][MAXD], K[7][MAXD];
  tsit5_stages(f, y, p, dt, S, K, NULL);
  const double a[7][6] = {
      {0, 0, 0, 0, 0, 0},
      {A21, 0, 0, 0, 0, 0},
      {A31, A32, 0, 0, 0, 0},
      {A41, A42, A43, 0, 0, 0},
      {A51, A52, A53, A54, 0, 0},
      {A61, A62, A63, A64, A65, 0},
      {B1, B2, B3, B4, B5, B6}};
  const double b[7] = {B1, B2, B3, B4, B5, B6, B7};
  double kb[7][MAXD], ybar[MAXD], sb[MAXD], g[MAXD];
  for (int i = 0; i < D; ++i) { ybar[i] = lam[i]; g[i] = dt * lam[i]; }
  for (int m = 0; m < 7; ++m)
    for (int i = 0; i < D; ++i) kb[m][i] = b[m] * g[i];
  for (int m = 6; m >= 0; --m) {
    for (int i = 0; i < D; ++i) sb[i] = 0.0;
    rhs_vjp(f, S[m], p, kb[m], sb, gp);
    for (int i = 0; i < D; ++i) ybar[i] += sb[i];
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < D; ++i) kb[j][i] += a[m][j] * (dt * sb[i]);
  }
  for (int i = 0; i < D; ++i) lam[i] = ybar[i];
}

/* ---------------------------------------------------------------------------------- */
/* Rosenbrock23                                                                       */
/* ---------------------------------------------------------------------------------- */

static void ros_init(void) {
  if (ROS_D != 0.0) return;
  ROS_D = 1.0 / (2.0 + sqrt(2.0));
  ROS_E32 = 6.0 + sqrt(2.0);
  ROS_EXP = -1.0 / 3.0;
}

/* _gauss_solve (_warp_rosenbrock.py:346-381): partial pivot, division, fresh copy. */
static void gauss_solve(const double* A, const double* b, double* out, int D) {
  double M[MAXD * MAXD], x[MAXD];
  memcpy(M, A, sizeof(double) * D * D);
  memcpy(x, b, sizeof(double) * D);
  for (int col = 0; col < D; ++col) {
    int piv = col;
    double big = fabs(M[col * D + col]);
    for (int r = col + 1; r < D; ++r) {
      double v = fabs(M[r * D + col]);
      if (v > big) { big = v; piv = r; }
    }
    if (piv != col) {
      for (int c = 0; c < D; ++c) {
        double tmp = M[col * D + c];
        M[col * D + c] = M[piv * D + c];
        M[piv * D + c] = tmp;
      }
      double tb = x[col];
      x[col] = x[piv];
      x[piv] = tb;
    }
    for (int r = col + 1; r < D; ++r) {
      double factor = M[r * D + col] / M[col * D + col];
      for (int c = col; c < D; ++c) M[r * D + c] = M[r * D + c] - factor * M[col * D + c];
      x[r] = x[r] - factor * x[col];
    }
  }
  for (int ii = 0; ii < D; ++ii) {
    int i = D - 1 - ii;
    double s = x[i];
    for (int c = i + 1; c < D; ++c) s = s - M[i * D + c] * out[c];
    out[i] = s / M[i * D + i];
  }
}

static void build_W(const field_t* f, const double* y, const double* p, double h, double* W) {
  const int D = f->D;
  double J[MAXD * MAXD];
  jac(f, y, p, J);
  for (int i = 0; i < D; ++i) {
    for (int c = 0; c < D; ++c) W[i * D + c] = -ROS_D * h * J[i * D + c];
    W[i * D + i] = W[i * D + i] + 1.0;
  }
}

static int ros23_one(const field_t* f, const double* y0, const double* p, double t0,
                     double t1, double rtol, double atol, double dt0, int max_steps, int cap,
                     double* dts, double* yf, int* n_acc, int* n_rej) {
  const int D = f->D;
  double y[MAXD], W[MAXD * MAXD], F0[MAXD], F1[MAXD], F2[MAXD], k1[MAXD], k2[MAXD],
      k3[MAXD], s[MAXD], ynew[MAXD], ev[MAXD];
  for (int i = 0; i < D; ++i) y[i] = y0[i];
  double t = t0, dt = dt0;
  int acc = 0, rej = 0, status = 0;
  for (int it = 0; it < max_steps; ++it) {
    if (t >= t1) break;
    double h = (t1 - t < dt) ? (t1 - t) : dt;
    build_W(f, y, p, h, W);
    rhs(f, y, p, F0);
    gauss_solve(W, F0, k1, D);
    for (int i = 0; i < D; ++i) s[i] = y[i] + 0.5 * h * k1[i];
    rhs(f, s, p, F1);
    for (int i = 0; i < D; ++i) s[i] = F1[i] - k1[i];
    gauss_solve(W, s, k2, D);
    for (int i = 0; i < D; ++i) k2[i] = k2[i] + k1[i];
    for (int i = 0; i < D; ++i) ynew[i] = y[i] + h * k2[i];
    rhs(f, ynew, p, F2);
    for (int i = 0; i < D; ++i) s[i] = F2[i] - ROS_E32 * (k2[i] - F1[i]) - 2.0 * (k1[i] - F0[i]);
    gauss_solve(W, s, k3, D);
    for (int i = 0; i < D; ++i) ev[i] = (h / 6.0) * (k1[i] - 2.0 * k2[i] + k3[i]);
    double err = wrms(ev, y, ynew, rtol, atol, D);
    if (err <= 1.0) {
      if (acc >= cap) { status = 3; break; }
      t = t + h;
      for (int i = 0; i < D; ++i) y[i] = ynew[i];
      dts[acc] = h;
      ++acc;
    } else {
      ++rej;
    }
    dt = controller(err, h, ROS_EXP);
  }
  if (status == 0 && !(t >= t1)) status = 1;
  for (int i = 0; i < D; ++i) yf[i] = y[i];
  *n_acc = acc;
  *n_rej = rej;
  return status;
}

/* rosenbrock23_step (rosenbrock23_step.py:47-66) with the analytic Jacobian. */
static void ros23_step(const field_t* f, const double* y, const double* p, double dt,
                       double* ynext) {
  const int D = f->D;
  double W[MAXD * MAXD], F0[MAXD], F1[MAXD], k1[MAXD], k2[MAXD], s[MAXD];
  build_W(f, y, p, dt, W);
  rhs(f, y, p, F0);
  gauss_solve(W, F0, k1, D);
  for (int i = 0; i < D; ++i) s[i] = y[i] + 0.5 * dt * k1[i];
  rhs(f, s, p, F1);
  for (int i = 0; i < D; ++i) s[i] = F1[i] - k1[i];
  gauss_solve(W, s, k2, D);
  for (int i = 0; i < D; ++i) k2[i] = k2[i] + k1[i];
  for (int i = 0; i < D; ++i) ynext[i] = y[i] + dt * k2[i];
}

/* Reverse of ros23_step: lam <- (dy'/dy)^T lam, gp += (dy'/dp)^T lam. */
static void ros23_step_vjp(const field_t* f, const double* y, const double* p, double dt,
                           double* lam, double* gp) {
  const int D = f->D;
  double W[MAXD * MAXD], WT[MAXD * MAXD], F0[MAXD], F1[MAXD], k1[MAXD], k2p[MAXD],
      s1[MAXD], r2[MAXD];
  build_W(f, y, p, dt, W);
  for (int i = 0; i < D; ++i)
    for (int c = 0; c < D; ++c) WT[i * D + c] = W[c * D + i];
  rhs(f, y, p, F0);
  gauss_solve(W, F0, k1, D);
  for (int i = 0; i < D; ++i) s1[i] = y[i] + 0.5 * dt * k1[i];
  rhs(f, s1, p, F1);
  for (int i = 0; i < D; ++i) r2[i] = F1[i] - k1[i];
  gauss_solve(W, r2, k2p, D);

  double ybar[MAXD], k2b[MAXD], k1b[MAXD], r2b[MAXD], F1b[MAXD], s1b[MAXD], r1b[MAXD];
  double Wb[MAXD * MAXD], G[MAXD * MAXD];
  for (int i = 0; i < D; ++i) { ybar[i] = lam[i]; k2b[i] = dt * lam[i]; }
  /* k2 = k2' + k1 */
  for (int i = 0; i < D; ++i) k1b[i] = k2b[i];
  /* W k2' = r2 */
  gauss_solve(WT, k2b, r2b, D);
  for (int i = 0; i < D; ++i)
    for (int c = 0; c < D; ++c) Wb[i * D + c] = -r2b[i] * k2p[c];
  /* r2 = F1 - k1 */
  for (int i = 0; i < D; ++i) { F1b[i] = r2b[i]; k1b[i] -= r2b[i]; s1b[i] = 0.0; }
  /* F1 = f(s1), s1 = y + 0.5*dt*k1 */
  rhs_vjp(f, s1, p, F1b, s1b, gp);
  for (int i = 0; i < D; ++i) { ybar[i] += s1b[i]; k1b[i] += 0.5 * dt * s1b[i]; }
  /* W k1 = F0 */
  gauss_solve(WT, k1b, r1b, D);
  for (int i = 0; i < D; ++i)
    for (int c = 0; c < D; ++c) Wb[i * D + c] += -r1b[i] * k1[c];
  /* F0 = f(y) */
  rhs_vjp(f, y, p, r1b, ybar, gp);
  /* W = I - d*dt*J(y,p) */
  for (int a = 0; a < D * D; ++a) G[a] = -ROS_D * dt * Wb[a];
  jac_contract_grad(f, y, p, G, ybar, gp);
  for (int i = 0; i < D; ++i) lam[i] = ybar[i];
}

/* ---------------------------------------------------------------------------------- */
/* exported batch entry points                                                        */
/* ---------------------------------------------------------------------------------- */

int gso_field_info(int code, int* D, int* P) {
  field_t f;
  if (field_make(code, &f)) return -1;
  *D = f.D;
  *P = f.P;
  return 0;
}

/* Minimal work-sharing loop over trajectories on host threads (pthreads; chunks of 16
 * handed out through an atomic counter). nthreads <= 0 uses one thread. */
typedef struct {
  long n;
  atomic_long next;
  void (*body)(long j, void* ctx);
  void* ctx;
} pfor_t;

static void* pfor_worker(void* arg) {
  pfor_t* w = (pfor_t*)arg;
  for (;;) {
    long j0 = atomic_fetch_add(&w->next, 16);
    if (j0 >= w->n) break;
    long j1 = j0 + 16 < w->n ? j0 + 16 : w->n;
    for (long j = j0; j < j1; ++j) w->body(j, w->ctx);
  }
  return NULL;
}

static void parallel_for(long n, int nthreads, void (*body)(long, void*), void* ctx) {
  pfor_t w;
  w.n = n;
  atomic_init(&w.next, 0);
  w.body = body;
  w.ctx = ctx;
  if (nthreads <= 1 || n <= 16) {
    pfor_worker(&w);
    return;
  }
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  int started = 0;
  for (int i = 0; i < nthreads - 1; ++i)
    if (pthread_create(&th[started], NULL, pfor_worker, &w) == 0) ++started;
  pfor_worker(&w);
  for (int i = 0; i < started; ++i) pthread_join(th[i], NULL);
}

typedef struct {
  int method;
  field_t f;
  const double *y0, *p, *t1v, *dts, *ybar;
  double t0, t1, rtol, atol, dt0;
  int max_steps, cap;
  long S;
  double *dts_out, *yf, *gy0, *gp;
  int *n_acc, *n_rej, *status;
  atomic_int err;
} job_t;

static void record_body(long j, void* ctx) {
  job_t* a = (job_t*)ctx;
  const int D = a->f.D, P = a->f.P;
  double t1j = a->t1v ? a->t1v[j] : a->t1;
  double dt0j = a->dt0 > 0.0 ? a->dt0 : (t1j - a->t0) / 100.0;
  double* row = a->dts_out + (size_t)j * (size_t)a->cap;
  memset(row, 0, sizeof(double) * (size_t)a->cap);
  if (a->method == 0)
    a->status[j] = tsit5_one(&a->f, a->y0 + j * D, a->p + j * P, a->t0, t1j, a->rtol, a->atol,
                             dt0j, a->max_steps, a->cap, row, a->yf + j * D, a->n_acc + j,
                             a->n_rej + j);
  else
    a->status[j] = ros23_one(&a->f, a->y0 + j * D, a->p + j * P, a->t0, t1j, a->rtol, a->atol,
                             dt0j, a->max_steps, a->cap, row, a->yf + j * D, a->n_acc + j,
                             a->n_rej + j);
}

/* method: 0 = tsit5, 1 = rosenbrock23.  dts: n*cap row-major, zero padded past n_acc.
 * t1v: per-trajectory end times (NULL -> t1).  dt0 <= 0 -> (t1_j - t0)/100. */
int gso_record(int method, int code, long n, const double* y0, const double* p, double t0,
               const double* t1v, double t1, double rtol, double atol, double dt0,
               int max_steps, int cap, double* dts, double* yf, int* n_acc, int* n_rej,
               int* status, int nthreads) {
  job_t a;
  memset(&a, 0, sizeof a);
  if (field_make(code, &a.f)) return -1;
  init_tableau();
  ros_init();
  a.method = method; a.y0 = y0; a.p = p; a.t0 = t0; a.t1v = t1v; a.t1 = t1;
  a.rtol = rtol; a.atol = atol; a.dt0 = dt0; a.max_steps = max_steps; a.cap = cap;
  a.dts_out = dts; a.yf = yf; a.n_acc = n_acc; a.n_rej = n_rej; a.status = status;
  parallel_for(n, nthreads, record_body, &a);
  return 0;
}

static void replay_body(long j, void* ctx) {
  job_t* a = (job_t*)ctx;
  const int D = a->f.D, P = a->f.P;
  double y[MAXD], yn[MAXD], S7[7][MAXD], K7[7][MAXD];
  for (int i = 0; i < D; ++i) y[i] = a->y0[j * D + i];
  for (long s = 0; s < a->S; ++s) {
    double dt = a->dts[j * a->S + s];
    if (a->method == 0)
      tsit5_stages(&a->f, y, a->p + j * P, dt, S7, K7, yn);
    else
      ros23_step(&a->f, y, a->p + j * P, dt, yn);
    for (int i = 0; i < D; ++i) y[i] = yn[i];
  }
  for (int i = 0; i < D; ++i) a->yf[j * D + i] = y[i];
}

/* Replay of padded dts [n,S] (warp_replay.py:30-55 / :267-293). */
int gso_replay(int method, int code, long n, const double* y0, const double* p, double t0,
               const double* dts, long S, double* yf, int nthreads) {
  job_t a;
  memset(&a, 0, sizeof a);
  if (field_make(code, &a.f)) return -1;
  init_tableau();
  ros_init();
  a.method = method; a.y0 = y0; a.p = p; a.t0 = t0; a.dts = dts; a.S = S; a.yf = yf;
  parallel_for(n, nthreads, replay_body, &a);
  return 0;
}

static void vjp_body(long j, void* ctx) {
  job_t* a = (job_t*)ctx;
  const int D = a->f.D, P = a->f.P;
  const long S = a->S;
  long len = 0;
  for (long s = 0; s < S; ++s)
    if (a->dts[j * S + s] != 0.0) len = s + 1; /* zero steps past len are identities */
  double* hist = (double*)malloc(sizeof(double) * (size_t)(len + 1) * (size_t)D);
  if (!hist) {
    atomic_store(&a->err, -2);
    return;
  }
  double y[MAXD], yn[MAXD], S7[7][MAXD], K7[7][MAXD], lam[MAXD], gp[MAXP];
  for (int i = 0; i < D; ++i) y[i] = a->y0[j * D + i];
  for (long s = 0; s < len; ++s) {
    memcpy(hist + s * D, y, sizeof(double) * D);
    double dt = a->dts[j * S + s];
    if (a->method == 0)
      tsit5_stages(&a->f, y, a->p + j * P, dt, S7, K7, yn);
    else
      ros23_step(&a->f, y, a->p + j * P, dt, yn);
    for (int i = 0; i < D; ++i) y[i] = yn[i];
  }
  for (int i = 0; i < D; ++i) lam[i] = a->ybar[j * D + i];
  for (int k = 0; k < P; ++k) gp[k] = 0.0;
  for (long s = len - 1; s >= 0; --s) {
    double dt = a->dts[j * S + s];
    if (a->method == 0)
      tsit5_step_vjp(&a->f, hist + s * D, a->p + j * P, dt, lam, gp);
    else
      ros23_step_vjp(&a->f, hist + s * D, a->p + j * P, dt, lam, gp);
  }
  free(hist);
  if (a->gy0)
    for (int i = 0; i < D; ++i) a->gy0[j * D + i] = lam[i];
  if (a->gp)
    for (int k = 0; k < P; ++k) a->gp[j * P + k] = gp[k];
}

/* Gradient of sum(ybar * replay(y0, p, dts)) w.r.t. y0 and p (frozen dts). gy0/gp may be
 * NULL. All intermediate states are kept (oracle: memory is not a concern). */
int gso_replay_vjp(int method, int code, long n, const double* y0, const double* p,
                   double t0, const double* dts, long S, const double* ybar, double* gy0,
                   double* gp_out, int nthreads) {
  job_t a;
  memset(&a, 0, sizeof a);
  if (field_make(code, &a.f)) return -1;
  init_tableau();
  ros_init();
  a.method = method; a.y0 = y0; a.p = p; a.t0 = t0; a.dts = dts; a.S = S; a.ybar = ybar;
  a.gy0 = gy0; a.gp = gp_out;
  atomic_init(&a.err, 0);
  parallel_for(n, nthreads, vjp_body, &a);
  return atomic_load(&a.err);
}

/* The eight Tsit5 error weights as this file evaluates them (checked against the
 * reference module's values in the tests). */
void gso_tsit5_error_weights(double* out7) {
  init_tableau();
  out7[0] = E1; out7[1] = E2; out7[2] = E3; out7[3] = E4;
  out7[4] = E5; out7[5] = E6; out7[6] = E7;
}
