/*
 * esr_cpu.c -- multi-threaded C restatement of the oracle's SRK2 step.
 *
 * TEST INFRASTRUCTURE ONLY: the timed CPU baseline (bench.py cpu_baseline
 * and --impl reference) and a cross-check of the NumPy oracle. It follows
 * oracle/euler_oracle.py, which restates euler/jax_fvm/src/euler_solver.py
 * and helper.py of EulerSR: BC ghosts (helper.py:168-256), LSQ gradient with
 * a 2x2 solve per cell (helper.py:136-153), Venkatakrishnan limiter with the
 * min over three faces (euler_solver.py:36-67), MUSCL, first order on
 * boundary faces (euler_solver.py:69-98), HLLC assembled as Fc - (Fc - F)
 * (euler_solver.py:273-420), sponge (helper.py:262-295), SRK2
 * (euler_solver.py:635-643). Compiled once per precision (REAL = double or
 * float); cells are processed in parallel with OpenMP.
 *
 * Geometry comes from the caller, per cell slot k: neighbour (or -1), kind
 * (0 interior, 2 wall, 3 inlet, 4 outlet), normal, face length, face
 * midpoint offset from the barycentre, LSQ offset (neighbour barycentre or
 * twice the face offset), and the neighbour's offset to the same midpoint.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif
#ifndef SUFFIX
#define SUFFIX f64
#endif
#define CAT2(a, b) a##_##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

typedef REAL R;

typedef struct {
  int n;
  const int* nbr;      /* n*3 */
  const int* kind;     /* n*3 */
  const R* nrm;        /* n*3*2 */
  const R* s;          /* n*3 */
  const R* dxf;        /* n*3*2  midpoint - barycentre */
  const R* dxl;        /* n*3*2  LSQ offsets */
  const R* dxn;        /* n*3*2  midpoint - neighbour barycentre */
  const R* area;       /* n */
  const R* sigma;      /* n  sponge strength * blend^3 */
  R gamma, gm1;
  R eps_lim;
  R inlet[4];
} Mesh;

static inline void prim(const R* W, R gm1, R* P) {
  const R r = W[0], u = W[1] / r, v = W[2] / r;
  P[0] = r; P[1] = u; P[2] = v;
  P[3] = (W[3] - (R)0.5 * r * (u * u + v * v)) * gm1;
}
static inline void cons(const R* P, R gm1, R* W) {
  const R r = P[0], u = P[1], v = P[2];
  W[0] = r; W[1] = r * u; W[2] = r * v;
  W[3] = P[3] / gm1 + (R)0.5 * r * (u * u + v * v);
}
static inline void ghost(const Mesh* m, int kind, const R* Wc, R nx, R ny, R* G) {
  if (kind == 2) {
    R P[4], Q[4];
    const R g14 = (R)(1.4 - 1.0);
    prim(Wc, g14, P);
    const R vn = P[1] * nx + P[2] * ny;
    Q[0] = P[0]; Q[1] = P[1] - (R)2 * vn * nx; Q[2] = P[2] - (R)2 * vn * ny; Q[3] = P[3];
    cons(Q, g14, G);
  } else if (kind == 3) {
    memcpy(G, m->inlet, 4 * sizeof(R));
  } else {
    memcpy(G, Wc, 4 * sizeof(R));
  }
}
static inline R venk(R a, R b) { return (a * a + (R)2 * a * b) / (a * a + (R)2 * b * b + a * b + (R)1e-7); }

static void hllc(const R* WL, const R* PL, const R* WR, const R* PR, R nx, R ny, R g, R* F) {
  const R rL = PL[0], uL = PL[1], vL = PL[2], pL = PL[3];
  const R rR = PR[0], uR = PR[1], vR = PR[2], pR = PR[3];
  const R unL = uL * nx + vL * ny, unR = uR * nx + vR * ny;
  const R tx = -ny, ty = nx;
  const R utL = uL * tx + vL * ty, utR = uR * tx + vR * ty;
  const R aL = sqrt(fabs(g * pL / rL)), aR = sqrt(fabs(g * pR / rR));
  R SL = fmin(unL - aL, unR - aR), SR = fmax(unL + aL, unR + aR);
  if (SL == SR) SL = SL - (R)1e-6;
  if (SL == SR) SR = SR + (R)1e-6;
  const R EL = WL[3], ER = WR[3];
  const R FL[4] = {rL * unL, rL * uL * unL + pL * nx, rL * vL * unL + pL * ny, (EL + pL) * unL};
  const R FR[4] = {rR * unR, rR * uR * unR + pR * nx, rR * vR * unR + pR * ny, (ER + pR) * unR};
  R den = rL * (SL - unL) - rR * (SR - unR);
  if (den == (R)0) den = (R)1e-12;
  const R Ss = (pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR)) / den;
  const R Ps = (R)0.5 * ((pL + rL * (SL - unL) * (Ss - unL)) + (pR + rR * (SR - unR) * (Ss - unR)));
  R H[4];
  if (SL >= 0) {
    memcpy(H, FL, sizeof(H));
  } else if (SL <= 0 && Ss >= 0) {
    const R rs = rL * (SL - unL) / (SL - Ss);
    const R U[4] = {rs, rs * (Ss * nx + utL * tx), rs * (Ss * ny + utL * ty),
                    ((SL - unL) * EL - pL * unL + Ps * Ss) / (SL - Ss)};
    for (int q = 0; q < 4; ++q) H[q] = FL[q] + SL * (U[q] - WL[q]);
  } else if (Ss <= 0 && SR >= 0) {
    const R rs = rR * (SR - unR) / (SR - Ss);
    const R U[4] = {rs, rs * (Ss * nx + utR * tx), rs * (Ss * ny + utR * ty),
                    ((SR - unR) * ER - pR * unR + Ps * Ss) / (SR - Ss)};
    for (int q = 0; q < 4; ++q) H[q] = FR[q] + SR * (U[q] - WR[q]);
  } else {
    memcpy(H, FR, sizeof(H));
  }
  for (int q = 0; q < 4; ++q) {
    const R Fc = (R)0.5 * (FL[q] + FR[q]);
    F[q] = Fc - (Fc - H[q]);
  }
}

/* residual R = sum_k F_k s_k / area - sigma (inlet - W) */
static void residual(const Mesh* m, const R* W, R* Pc, R* G, R* phi, R* Res) {
  const int n = m->n;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < n; ++c) {
    const R* Wc = W + 4 * c;
    R P[4], Pk[3][4];
    prim(Wc, m->gm1, P);
    for (int k = 0; k < 3; ++k) {
      R Wk[4];
      const int kind = m->kind[3 * c + k];
      if (kind == 0) memcpy(Wk, W + 4 * m->nbr[3 * c + k], sizeof(Wk));
      else ghost(m, kind, Wc, m->nrm[6 * c + 2 * k], m->nrm[6 * c + 2 * k + 1], Wk);
      prim(Wk, m->gm1, Pk[k]);
    }
    R a11 = 0, a12 = 0, a22 = 0;
    R bx[4] = {0, 0, 0, 0}, by[4] = {0, 0, 0, 0};
    for (int k = 0; k < 3; ++k) {
      const R dx = m->dxl[6 * c + 2 * k], dy = m->dxl[6 * c + 2 * k + 1];
      const R w = (R)1 / (dx * dx + dy * dy);
      a11 += w * dx * dx; a12 += w * dx * dy; a22 += w * dy * dy;
      for (int v = 0; v < 4; ++v) {
        const R d = Pk[k][v] - P[v];
        bx[v] += w * d * dx;
        by[v] += w * d * dy;
      }
    }
    const R det = a11 * a22 - a12 * a12;
    for (int v = 0; v < 4; ++v) {
      const R gx = (a22 * bx[v] - a12 * by[v]) / det, gy = (a11 * by[v] - a12 * bx[v]) / det;
      G[8 * c + 2 * v] = gx;
      G[8 * c + 2 * v + 1] = gy;
      R mn = P[v], mx = P[v];
      for (int k = 0; k < 3; ++k) { mn = fmin(mn, Pk[k][v]); mx = fmax(mx, Pk[k][v]); }
      R ph = 0;
      for (int k = 0; k < 3; ++k) {
        const R D = m->dxf[6 * c + 2 * k] * gx + m->dxf[6 * c + 2 * k + 1] * gy;
        R p = 1;
        if (D > m->eps_lim) p = venk(mx - P[v], D);
        else if (D < -m->eps_lim) p = venk(mn - P[v], D);
        ph = (k == 0) ? p : fmin(ph, p);
      }
      phi[4 * c + v] = ph;
      Pc[4 * c + v] = P[v];
    }
  }
#pragma omp parallel for schedule(static)
  for (int c = 0; c < n; ++c) {
    const R* Wc = W + 4 * c;
    R acc[4] = {0, 0, 0, 0};
    for (int k = 0; k < 3; ++k) {
      const int kind = m->kind[3 * c + k];
      const R nx = m->nrm[6 * c + 2 * k], ny = m->nrm[6 * c + 2 * k + 1];
      R qL[4], qR[4], WL[4], WR[4], PL[4], PR[4], F[4];
      if (kind == 0) {
        const int j = m->nbr[3 * c + k];
        for (int v = 0; v < 4; ++v) {
          const R gx = G[8 * c + 2 * v], gy = G[8 * c + 2 * v + 1];
          qL[v] = Pc[4 * c + v] + phi[4 * c + v] * (m->dxf[6 * c + 2 * k] * gx + m->dxf[6 * c + 2 * k + 1] * gy);
          const R hx = G[8 * j + 2 * v], hy = G[8 * j + 2 * v + 1];
          qR[v] = Pc[4 * j + v] + phi[4 * j + v] * (m->dxn[6 * c + 2 * k] * hx + m->dxn[6 * c + 2 * k + 1] * hy);
        }
      } else {
        R Gh[4];
        ghost(m, kind, Wc, nx, ny, Gh);
        prim(Gh, m->gm1, qR);
        for (int v = 0; v < 4; ++v) qL[v] = Pc[4 * c + v];
      }
      cons(qL, m->gm1, WL);
      cons(qR, m->gm1, WR);
      prim(WL, m->gm1, PL);
      prim(WR, m->gm1, PR);
      hllc(WL, PL, WR, PR, nx, ny, m->gamma, F);
      for (int q = 0; q < 4; ++q) acc[q] += m->s[3 * c + k] * F[q];
    }
    for (int q = 0; q < 4; ++q)
      Res[4 * c + q] = acc[q] / m->area[c] - m->sigma[c] * (m->inlet[q] - Wc[q]);
  }
}

/* nsteps SRK2 steps of one case in place; scratch is allocated per call */
int FN(esr_cpu_srk2)(int n, const int* nbr, const int* kind, const R* nrm, const R* s, const R* dxf, const R* dxl,
                     const R* dxn, const R* area, const R* sigma, R gamma, const R* inlet, R dt, int nsteps, R* W) {
  Mesh m = {n, nbr, kind, nrm, s, dxf, dxl, dxn, area, sigma, gamma, (R)(gamma - 1.0),
            sizeof(R) == 8 ? (R)1e-12 : (R)1e-7, {inlet[0], inlet[1], inlet[2], inlet[3]}};
  R* W1 = (R*)malloc(sizeof(R) * 4 * n);
  R* Pc = (R*)malloc(sizeof(R) * 4 * n);
  R* G = (R*)malloc(sizeof(R) * 8 * n);
  R* ph = (R*)malloc(sizeof(R) * 4 * n);
  R* Res = (R*)malloc(sizeof(R) * 4 * n);
  if (!W1 || !Pc || !G || !ph || !Res) {
    free(W1); free(Pc); free(G); free(ph); free(Res);
    return 1;
  }
  for (int it = 0; it < nsteps; ++it) {
    residual(&m, W, Pc, G, ph, Res);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < 4 * n; ++i) W1[i] = W[i] - dt * Res[i];
    residual(&m, W1, Pc, G, ph, Res);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < 4 * n; ++i) W[i] = (R)0.5 * (W[i] + W1[i] - dt * Res[i]);
  }
  free(W1); free(Pc); free(G); free(ph); free(Res);
  return 0;
}

/* nsteps SRK2 steps with the per-cell CFL step of the state at the start of
 * each step (the local-time-step option: dt_c = cfl * area_c / sum_k
 * (c + |u.n_k|) s_k, helper.py:8-18 per cell), as oracle/euler_oracle.py
 * time_step_srk2_local */
int FN(esr_cpu_srk2_local)(int n, const int* nbr, const int* kind, const R* nrm, const R* s, const R* dxf,
                           const R* dxl, const R* dxn, const R* area, const R* sigma, R gamma, const R* inlet, R cfl,
                           int nsteps, R* W) {
  Mesh m = {n, nbr, kind, nrm, s, dxf, dxl, dxn, area, sigma, gamma, (R)(gamma - 1.0),
            sizeof(R) == 8 ? (R)1e-12 : (R)1e-7, {inlet[0], inlet[1], inlet[2], inlet[3]}};
  R* W1 = (R*)malloc(sizeof(R) * 4 * n);
  R* Pc = (R*)malloc(sizeof(R) * 4 * n);
  R* G = (R*)malloc(sizeof(R) * 8 * n);
  R* ph = (R*)malloc(sizeof(R) * 4 * n);
  R* Res = (R*)malloc(sizeof(R) * 4 * n);
  R* dt = (R*)malloc(sizeof(R) * n);
  if (!W1 || !Pc || !G || !ph || !Res || !dt) {
    free(W1); free(Pc); free(G); free(ph); free(Res); free(dt);
    return 1;
  }
  for (int it = 0; it < nsteps; ++it) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < n; ++c) {
      R P[4];
      prim(W + 4 * c, m.gm1, P);
      const R cel = sqrt(fabs(gamma * P[3] / P[0]));
      R lam = 0;
      for (int k = 0; k < 3; ++k) {
        const R un = P[1] * nrm[6 * c + 2 * k] + P[2] * nrm[6 * c + 2 * k + 1];
        lam += (cel + fabs(un)) * s[3 * c + k];
      }
      dt[c] = area[c] / lam * cfl;
    }
    residual(&m, W, Pc, G, ph, Res);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < 4 * n; ++i) W1[i] = W[i] - dt[i / 4] * Res[i];
    residual(&m, W1, Pc, G, ph, Res);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < 4 * n; ++i) W[i] = (R)0.5 * (W[i] + W1[i] - dt[i / 4] * Res[i]);
  }
  free(W1); free(Pc); free(G); free(ph); free(Res); free(dt);
  return 0;
}
