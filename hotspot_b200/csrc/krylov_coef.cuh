// krylov_coef.cuh -- coefficient algebra of the Krylov-form RK4 (shared by
// the single-model kernel, rk4_krylov.cu, and the batched kernel,
// rk4_batch.cu).
//
// Within a sampling interval the slope is affine, f(T) = L T + c, so every
// stage of the reference's step-doubling RK4 (RCutil.c:440-640) is a
// polynomial in L applied to F = f(y).  Vectors are represented by their
// coefficients over the basis N_m = s_m L N_{m-1}, N_0 = F.
#pragma once

namespace hsb {

#define PMAX (KRY_DMAX + 8)   // coefficient array length

struct Coef {
  double c[PMAX];
  int n;                           // number of coefficients
};

// ---------------------------------------------------------------------------
// coefficient algebra over the basis N_m = (s L)^m F (one thread)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void c_one(Coef &p) {
  p.n = 1;
  p.c[0] = 1.0;
}
__device__ __forceinline__ void c_copy(Coef &d, const Coef &s) {
  d.n = s.n;
  for (int j = 0; j < s.n; j++) d.c[j] = s.c[j];
}
// w = L v: L N_m = N_{m+1} / s_{m+1}
__device__ __forceinline__ void c_lop(Coef &w, const Coef &v, const double *ps) {
  const int n = v.n + 1 < PMAX ? v.n + 1 : PMAX;
  w.c[0] = 0.0;
  for (int j = 1; j < n; j++) w.c[j] = v.c[j - 1] / ps[j];
  w.n = n;
}
// y += a x
__device__ __forceinline__ void c_axpy(Coef &y, double a, const Coef &x) {
  for (int j = y.n; j < x.n; j++) y.c[j] = 0.0;
  if (x.n > y.n) y.n = x.n;
  for (int j = 0; j < x.n; j++) y.c[j] += a * x.c[j];
}
// y_out - y of rk4_core(y, k1 = K, h) with f(y) = F = N_0 (RCutil.c:440-531)
__device__ inline void c_core(Coef &out, const Coef &K, double h, const double *s) {
  Coef t, k2, k3, k4;
  c_lop(t, K, s);
  c_one(k2);
  c_axpy(k2, h / 2.0, t);
  c_lop(t, k2, s);
  c_one(k3);
  c_axpy(k3, h / 2.0, t);
  c_lop(t, k3, s);
  c_one(k4);
  c_axpy(k4, h, t);
  int n = K.n;
  if (k2.n > n) n = k2.n;
  if (k3.n > n) n = k3.n;
  if (k4.n > n) n = k4.n;
  for (int j = 0; j < n; j++) {
    const double a1 = j < K.n ? K.c[j] : 0.0, a2 = j < k2.n ? k2.c[j] : 0.0;
    const double a3 = j < k3.n ? k3.c[j] : 0.0, a4 = j < k4.n ? k4.c[j] : 0.0;
    out.c[j] = h * (a1 + 2 * a2 + 2 * a3 + a4) / 6.0;
  }
  out.n = n;
}

// the attempt's polynomials (one thread): D = ytemp - y, F1 = f(t1), E = ytemp - t2;
// vectors not computed yet (index > dcomp) will be made with scale h
__device__ inline void kry_plan(Coef &E, Coef &D, Coef &F1, const Coef &K, double *ps, double h, int dcomp) {
  for (int m = dcomp + 1; m < PMAX; m++) ps[m] = h;
  const double *s = ps;
  Coef dh, d2;
  c_core(D, K, h, s);
  c_core(dh, K, h / 2.0, s);
  Coef t;
  c_lop(t, dh, s);
  c_one(F1);
  c_axpy(F1, 1.0, t);
  // second half step from t1 with k1 = f(t1): its f is F1 as well
  {
    Coef k2, k3, k4, u;
    const double hh = h / 2.0;
    c_lop(u, F1, s);
    c_copy(k2, F1);
    c_axpy(k2, hh / 2.0, u);
    c_lop(u, k2, s);
    c_copy(k3, F1);
    c_axpy(k3, hh / 2.0, u);
    c_lop(u, k3, s);
    c_copy(k4, F1);
    c_axpy(k4, hh, u);
    int n = k4.n;
    for (int j = 0; j < n; j++) {
      const double a1 = j < F1.n ? F1.c[j] : 0.0, a2 = j < k2.n ? k2.c[j] : 0.0;
      const double a3 = j < k3.n ? k3.c[j] : 0.0, a4 = k4.c[j];
      d2.c[j] = hh * (a1 + 2 * a2 + 2 * a3 + a4) / 6.0;
    }
    d2.n = n;
  }
  // E = D - (dh + d2); coefficients that cancel to rounding against their
  // own terms (the low orders, exactly zero in exact arithmetic when K = F)
  // are dropped, the degree stays that of d2
  c_copy(E, D);
  c_axpy(E, -1.0, dh);
  c_axpy(E, -1.0, d2);
  for (int j = 0; j < E.n; j++) {
    const double ref = fabs(j < D.n ? D.c[j] : 0.0) + fabs(j < dh.n ? dh.c[j] : 0.0) +
                       fabs(j < d2.n ? d2.c[j] : 0.0);
    if (fabs(E.c[j]) <= 1e-12 * ref) E.c[j] = 0.0;
  }
}


}  // namespace hsb
