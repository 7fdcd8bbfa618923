/* CPU restatement of the reference's hydro force path, FP64.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle.  The product never links this file;
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it,
 * as the checker.  Parity of this restatement against the reference's own
 * compiled functors (oracle/_ref, built from the reference headers) is pinned
 * by tests/test_oracle_pin.py and by the committed vectors in tests/golden/.
 *
 * Compiled with -ffp-contract=off: every FP32 expression below (cell index,
 * neighbour predicate, periodic wrap) is evaluated exactly as written, with
 * explicit fmaf where the GPU uses a fused multiply-add, so the pair SET is
 * bit-identical to the GPU's; all physics is then evaluated in FP64.
 */
#include "wcsph_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------------ */
/* Cubic spline, 3-D (kernel.h:27-55): H = 2h, s = r/H,
 *   W     = [(1-s)+^3 - 4 (1/2-s)+^3] * 16/(pi H^3)
 *   gradW = dr * [-3 (1-s)+^2 + 12 (1/2-s)+^2] * 16/(pi H^3) / (r H)          */
static inline double plus(double x) { return x > 0.0 ? x : 0.0; }

double orc_W(double r, double h) {
  const double H = 2.0 * h, s = r / H;
  const double a = plus(1.0 - s), b = plus(0.5 - s);
  return (a * a * a - 4.0 * b * b * b) * (16.0 / M_PI) / (H * H * H);
}

/* Returns g such that gradW(dr, h) = g * dr. */
double orc_gradW_scalar(double r, double h) {
  const double H = 2.0 * h, s = r / H;
  const double a = plus(1.0 - s), b = plus(0.5 - s);
  return (-3.0 * a * a + 12.0 * b * b) * (16.0 / M_PI) / (H * H * H) / (r * H);
}

/* Tait / Murnaghan EoS (EoS.h:75-90): B = c0^2 rho0 / gamma,
 *   P = max(B ((rho/rho0)^gamma - 1), 0),  c = sqrt(max(B gamma/rho0 (rho/rho0)^(gamma-1), 1e-16)). */
void orc_eos(int n, const double* dens, double* pres, double* snds, double gamma, double rho0, double c0) {
  const double B = c0 * c0 * rho0 / gamma;
  for (int i = 0; i < n; ++i) {
    const double x = dens[i] / rho0;
    pres[i] = fmax(B * (pow(x, gamma) - 1.0), 0.0);
    snds[i] = sqrt(fmax(B * gamma / rho0 * pow(x, gamma - 1.0), 1.0e-16));
  }
}

/* ------------------------------------------------------------------------ */
/* One pair contribution, shared by walk and neighbour modes.
 * Restates force.h:40-54 (ref CPU) and kernel.cu:253-273 (ref GPU): with
 * dr = r_i - r_j, dv = v_i - v_j,
 *   mu    = drdv < 0 ? hbar drdv / (r^2 + eps h_i h_j) : 0
 *   Pi    = (-alpha c_ij mu + beta mu^2) / rho_ij
 *   a_i  -= m_j (P_i/rho_i^2 + P_j/rho_j^2 + Pi) gradW
 *   a_i  += m_j 2 (nu_i + nu_j) (dr.gradW) / (rho_i + rho_j) / (r^2 + eps h_i h_j) dv
 *   divv -= m_j dv.gradW                                                     */
typedef struct { double acc[3], divv, vsig; } pair_acc;

static inline void pair_term(const orc_pair_params* pp, const double dr[3], const double dv[3], double hi, double hj,
                             double rhoi, double rhoj, double poi, double poj, double ci, double cj, double nui,
                             double nuj, double mj, pair_acc* A) {
  const double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
  if (r2 <= 0.0) return; /* force.h:42 */
  const double r = sqrt(r2);
  const double drdv = dr[0] * dv[0] + dr[1] * dv[1] + dr[2] * dv[2];
  const double cij = 0.5 * (ci + cj), rhoij = 0.5 * (rhoi + rhoj);
  const double den = r2 + pp->eps * hi * hj;
  const double mu = drdv < 0.0 ? 0.5 * (hi + hj) * drdv / den : 0.0;
  const double PI = (-pp->alpha * cij * mu + pp->beta * mu * mu) / rhoij;
  if (pp->vsig_mode == ORC_VSIG_SIGNAL) A->vsig = fmax(A->vsig, -mu);
  else A->vsig = fmax(A->vsig, mu);
  double g;
  if (pp->grad_mode == ORC_GRAD_SYM) g = 0.5 * (orc_gradW_scalar(r, hi) + orc_gradW_scalar(r, hj));
  else g = orc_gradW_scalar(r, 0.5 * (hi + hj));
  const double pterm = poi + poj + PI;
  const double visc = 2.0 * (nui + nuj) * (g * r2) / (rhoi + rhoj) / den;
  for (int k = 0; k < 3; ++k) A->acc[k] += mj * (-pterm * g * dr[k] + visc * dv[k]);
  A->divv += -mj * g * drdv;
}

/* FDPS multiwalk semantics (kernel.cu:241-280, force.h:34-59): each i of a
 * walk against every j of the walk.  out[] is fully written (the clear() of
 * class.h:68-72 is implied). */
void orc_hydro_walks(int n_walk, const int* ni_displ, const orc_epi_hydro* epi, const int* nj_displ,
                     const orc_epj_hydro* epj, orc_result_hydro* out, const orc_pair_params* pp) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int w = 0; w < n_walk; ++w) {
    for (int i = ni_displ[w]; i < ni_displ[w + 1]; ++i) {
      const orc_epi_hydro* I = &epi[i];
      pair_acc A = {{0, 0, 0}, 0, 0};
      const double poi = I->pres / (I->dens * I->dens);
      for (int j = nj_displ[w]; j < nj_displ[w + 1]; ++j) {
        const orc_epj_hydro* J = &epj[j];
        double dr[3], dv[3];
        for (int k = 0; k < 3; ++k) {
          dr[k] = I->pos[k] - J->pos[k];
          dv[k] = I->vel[k] - J->vel[k];
        }
        pair_term(pp, dr, dv, I->smth, J->smth, I->dens, J->dens, poi, J->pres / (J->dens * J->dens), I->snds,
                  J->snds, I->visc, J->visc, J->mass, &A);
      }
      for (int k = 0; k < 3; ++k) out[i].acc[k] = A.acc[k];
      out[i].dt = pp->c_cfl * I->smth / (I->snds + A.vsig); /* force.h:56 */
      out[i].div_v = A.divv / I->dens;                       /* force.h:57 */
    }
  }
}

/* Shepard filter over walks (force.h:12-29). */
void orc_filter_walks(int n_walk, const int* ni_displ, const double* epi, const int* nj_displ, const double* epj,
                      double* out_dens) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int w = 0; w < n_walk; ++w) {
    for (int i = ni_displ[w]; i < ni_displ[w + 1]; ++i) {
      const double* I = &epi[4 * i];
      double one = 0.0, sum = 0.0;
      for (int j = nj_displ[w]; j < nj_displ[w + 1]; ++j) {
        const double* J = &epj[5 * j];
        const double dx = I[0] - J[0], dy = I[1] - J[1], dz = I[2] - J[2];
        const double W = orc_W(sqrt(dx * dx + dy * dy + dz * dz), I[3]);
        one += W * J[4] / J[3];
        sum += J[4] * W;
      }
      out_dens[i] = sum / one;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Neighbour mode.  Cell of a particle, FP32 (the device computes the same):
 *   c = (int) floorf((x - lo) * (1/cell)), clamped to [0, ncell-1].          */
static inline int cell_of(float x, float lo, float inv, int n) {
  int c = (int)floorf((x - lo) * inv);
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

static inline uint32_t spread3(uint32_t v) { /* 10 bits -> every third bit */
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

static void inv_cells(const orc_config* cfg, float inv[3]) {
  for (int k = 0; k < 3; ++k) inv[k] = 1.0f / cfg->cell[k];
}

void orc_cells(int n, const float* pos4, const orc_config* cfg, int32_t* cxyz, uint32_t* key) {
  float inv[3];
  inv_cells(cfg, inv);
  for (int i = 0; i < n; ++i) {
    int c[3];
    for (int k = 0; k < 3; ++k) c[k] = cell_of(pos4[4 * i + k], cfg->lo[k], inv[k], cfg->ncell[k]);
    if (cxyz) {
      cxyz[3 * i] = c[0];
      cxyz[3 * i + 1] = c[1];
      cxyz[3 * i + 2] = c[2];
    }
    if (key) key[i] = spread3((uint32_t)c[0]) | (spread3((uint32_t)c[1]) << 1) | (spread3((uint32_t)c[2]) << 2);
  }
}

void orc_sort_perm(int n, const uint32_t* key, int32_t* perm) {
  /* LSD radix sort, 8-bit digits: stable, so ties keep their input order. */
  int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; ++i) perm[i] = i;
  for (int shift = 0; shift < 32; shift += 8) {
    size_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (int i = 0; i < n; ++i) cnt[((key[perm[i]] >> shift) & 0xffu) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (int i = 0; i < n; ++i) tmp[cnt[(key[perm[i]] >> shift) & 0xffu]++] = perm[i];
    memcpy(perm, tmp, sizeof(int32_t) * (size_t)n);
  }
  free(tmp);
}

/* CSR cell table over the linear cell index (x fastest), used only to find
 * candidates quickly; the pair set itself is defined by the predicate. */
typedef struct { int ncell; int* start; int* idx; int (*cxyz)[3]; } cell_table;

static void table_build(int n, const float* pos4, const orc_config* cfg, cell_table* T) {
  const int nx = cfg->ncell[0], ny = cfg->ncell[1], nz = cfg->ncell[2];
  T->ncell = nx * ny * nz;
  T->start = (int*)calloc((size_t)T->ncell + 1, sizeof(int));
  T->idx = (int*)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  T->cxyz = (int(*)[3])malloc(sizeof(int) * 3 * (size_t)(n > 0 ? n : 1));
  orc_cells(n, pos4, cfg, (int32_t*)T->cxyz, NULL);
  for (int i = 0; i < n; ++i) T->start[(T->cxyz[i][2] * ny + T->cxyz[i][1]) * nx + T->cxyz[i][0] + 1]++;
  for (int c = 0; c < T->ncell; ++c) T->start[c + 1] += T->start[c];
  int* fill = (int*)malloc(sizeof(int) * (size_t)T->ncell);
  memcpy(fill, T->start, sizeof(int) * (size_t)T->ncell);
  for (int i = 0; i < n; ++i) T->idx[fill[(T->cxyz[i][2] * ny + T->cxyz[i][1]) * nx + T->cxyz[i][0]]++] = i;
  free(fill);
}

static void table_free(cell_table* T) {
  free(T->start);
  free(T->idx);
  free(T->cxyz);
}

/* Periodic images.  A candidate j is visited through one of the 27 cells
 * around i's cell; when that cell index wraps past the box edge on an axis,
 * j is taken at its image x_j + s L with s = +1 (wrapped past the high edge)
 * or s = -1 (past the low edge).  The FP32 displacement is
 *   d = x_i - (x_j + s L)           (two rounded operations, as on the device)
 * With at least 3 cells of edge >= 2h per periodic axis this is the minimum
 * image of every in-support pair.  Neighbour entries carry the shifts:
 *   entry = j * 27 + (sx+1) + 3 (sy+1) + 9 (sz+1).                           */
#define ENC(j, sx, sy, sz) ((j) * 27 + ((sx) + 1) + 3 * ((sy) + 1) + 9 * ((sz) + 1))
static inline int ent_j(int e) { return e / 27; }
static inline void ent_s(int e, int s[3]) {
  const int c = e % 27;
  s[0] = c % 3 - 1;
  s[1] = (c / 3) % 3 - 1;
  s[2] = c / 9 - 1;
}

/* The neighbour predicate, FP32, exactly as the device evaluates it:
 *   r2 = fma(dz,dz, fma(dy,dy, dx*dx)),  in support <=> 0 < r2 < H2,
 *   H = 2*(float)h, H2 = H*H.                                                */
static inline int in_support(const float* pi, const float* pj, const float sh[3], float H2) {
  float d[3];
  for (int k = 0; k < 3; ++k) d[k] = pi[k] - (pj[k] + sh[k]);
  const float r2 = fmaf(d[2], d[2], fmaf(d[1], d[1], d[0] * d[0]));
  return r2 > 0.0f && r2 < H2;
}

static inline float support2(const orc_config* cfg) {
  const float H = 2.0f * (float)cfg->h;
  return H * H;
}

static int cmp_int(const void* a, const void* b) { return (*(const int*)a > *(const int*)b) - (*(const int*)a < *(const int*)b); }

/* Encoded in-support neighbours of i, ascending j. */
static int gather_neighbors(int i, const float* pos4, const orc_config* cfg, const cell_table* T, float H2, int* buf,
                            int cap) {
  const int nc[3] = {cfg->ncell[0], cfg->ncell[1], cfg->ncell[2]};
  float L[3];
  for (int k = 0; k < 3; ++k) L[k] = cfg->hi[k] - cfg->lo[k];
  int m = 0;
  const int* c = T->cxyz[i];
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        int q[3] = {c[0] + dx, c[1] + dy, c[2] + dz}, s[3] = {0, 0, 0};
        int skip = 0;
        for (int k = 0; k < 3; ++k) {
          if (q[k] < 0 || q[k] >= nc[k]) {
            if (!cfg->periodic) skip = 1;
            else if (q[k] < 0) q[k] += nc[k], s[k] = -1;
            else q[k] -= nc[k], s[k] = 1;
          }
        }
        if (skip) continue;
        const float sh[3] = {s[0] * L[0], s[1] * L[1], s[2] * L[2]};
        const int lin = (q[2] * nc[1] + q[1]) * nc[0] + q[0];
        for (int p = T->start[lin]; p < T->start[lin + 1]; ++p) {
          const int j = T->idx[p];
          if (in_support(&pos4[4 * i], &pos4[4 * j], sh, H2)) {
            if (m < cap) buf[m] = ENC(j, s[0], s[1], s[2]);
            ++m;
          }
        }
      }
  if (m <= cap) qsort(buf, (size_t)m, sizeof(int), cmp_int);
  return m;
}

#define NB_CAP 1024

int64_t orc_neighbors(int n, const float* pos4, const orc_config* cfg, int32_t* count, int32_t* list, int cap) {
  cell_table T;
  table_build(n, pos4, cfg, &T);
  const float H2 = support2(cfg);
  int64_t total = 0;
  int overflow = 0;
#pragma omp parallel for reduction(+ : total) reduction(| : overflow) schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    int buf[NB_CAP];
    const int m = gather_neighbors(i, pos4, cfg, &T, H2, buf, NB_CAP);
    if (count) count[i] = m;
    total += m;
    if (list) {
      if (m > cap || m > NB_CAP) overflow = 1;
      const int mm = m < cap ? m : cap;
      for (int k = 0; k < mm && k < NB_CAP; ++k) list[(int64_t)i * cap + k] = ent_j(buf[k]);
    }
  }
  table_free(&T);
  return overflow ? -1 : total;
}

/* Image offset s L (FP64) of a neighbour entry. */
static inline void image_offset(int e, const orc_config* cfg, double off[3]) {
  int s[3];
  ent_s(e, s);
  for (int a = 0; a < 3; ++a) off[a] = s[a] * ((double)cfg->hi[a] - (double)cfg->lo[a]);
}

/* FP64 displacement x_i - (x_j + s L) of FP32 positions. */
static inline void disp64(const float* pos4, int i, int e, const orc_config* cfg, double d[3]) {
  double off[3];
  image_offset(e, cfg, off);
  const int j = ent_j(e);
  for (int a = 0; a < 3; ++a) d[a] = (double)pos4[4 * i + a] - ((double)pos4[4 * j + a] + off[a]);
}

void orc_density(int n, const float* pos4, const float* dens_in, const orc_config* cfg, int shepard,
                 double* dens_out) {
  cell_table T;
  table_build(n, pos4, cfg, &T);
  const float H2 = support2(cfg);
  const double h = cfg->h, m = cfg->mass;
  const double W0 = orc_W(0.0, h);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    int buf[NB_CAP];
    const int cnt = gather_neighbors(i, pos4, cfg, &T, H2, buf, NB_CAP);
    /* self term first (FDPS gather lists contain i itself, force.h:16-20) */
    double sum = m * W0, one = shepard ? m / (double)dens_in[i] * W0 : 0.0;
    for (int k = 0; k < cnt && k < NB_CAP; ++k) {
      const int j = ent_j(buf[k]);
      double d[3];
      disp64(pos4, i, buf[k], cfg, d);
      const double W = orc_W(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), h);
      sum += m * W;
      if (shepard) one += m / (double)dens_in[j] * W;
    }
    dens_out[i] = shepard ? sum / one : sum;
  }
  table_free(&T);
}

void orc_hydro(int n, const float* pos4, const float* vel4, const float* dens, const float* pres, const float* snds,
               const orc_config* cfg, double* acc3, double* div_v, double* dt) {
  cell_table T;
  table_build(n, pos4, cfg, &T);
  const float H2 = support2(cfg);
  const double h = cfg->h, m = cfg->mass, nu = cfg->nu;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    int buf[NB_CAP];
    const int cnt = gather_neighbors(i, pos4, cfg, &T, H2, buf, NB_CAP);
    pair_acc A = {{0, 0, 0}, 0, 0};
    const double rhoi = dens[i], poi = (double)pres[i] / (rhoi * rhoi);
    for (int k = 0; k < cnt && k < NB_CAP; ++k) {
      const int j = ent_j(buf[k]);
      double dr[3], dv[3];
      disp64(pos4, i, buf[k], cfg, dr);
      for (int a = 0; a < 3; ++a) dv[a] = (double)vel4[4 * i + a] - (double)vel4[4 * j + a];
      const double rhoj = dens[j];
      pair_term(&cfg->pair, dr, dv, h, h, rhoi, rhoj, poi, (double)pres[j] / (rhoj * rhoj), snds[i], snds[j], nu, nu,
                m, &A);
    }
    for (int a = 0; a < 3; ++a) acc3[3 * i + a] = A.acc[a];
    div_v[i] = A.divv / rhoi;
    dt[i] = cfg->pair.c_cfl * h / ((double)snds[i] + A.vsig);
  }
  table_free(&T);
}

double orc_dt_global(int n, const double* acc3, const double* dt, const int32_t* type, double h, double nu) {
  double g = 1.0e30;
  for (int i = 0; i < n; ++i) {
    if (type[i]) continue; /* FREEZE particles do not limit dt (integral.h:6) */
    double t = 1.0e30;
    const double a = sqrt(acc3[3 * i] * acc3[3 * i] + acc3[3 * i + 1] * acc3[3 * i + 1] + acc3[3 * i + 2] * acc3[3 * i + 2]);
    t = fmin(0.25 * sqrt(h / a), t);
    if (nu > 0.0) t = fmin(0.125 * h * h / nu, t);
    g = fmin(g, fmin(dt[i], t));
  }
  return g;
}

/* ------------------------------------------------------------------------ */
/* FP64 full step.  Positions are rounded to FP32 only to decide the pair set
 * (so that the set matches the device's for the same starting state). */
static void force_pass(int n, const double* pos3, const double* vel3, double* dens, double* acc3, double* div_v,
                       double* dt_i, const orc_config* cfg, int do_density, int shepard) {
  float* p4 = (float*)malloc(sizeof(float) * 4 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    for (int a = 0; a < 3; ++a) p4[4 * i + a] = (float)pos3[3 * i + a];
    p4[4 * i + 3] = 0.0f;
  }
  cell_table T;
  table_build(n, p4, cfg, &T);
  const float H2 = support2(cfg);
  const double h = cfg->h, m = cfg->mass, nu = cfg->nu;
  int* cnts = (int*)malloc(sizeof(int) * (size_t)n);
  int* lists = (int*)malloc(sizeof(int) * (size_t)n * NB_CAP);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) cnts[i] = gather_neighbors(i, p4, cfg, &T, H2, &lists[(size_t)i * NB_CAP], NB_CAP);
  if (do_density) {
    double* nd = (double*)malloc(sizeof(double) * (size_t)n);
    const double W0 = orc_W(0.0, h);
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) {
      double sum = m * W0, one = m / dens[i] * W0;
      for (int k = 0; k < cnts[i]; ++k) {
        const int e = lists[(size_t)i * NB_CAP + k], j = ent_j(e);
        double d[3];
        image_offset(e, cfg, d);
        for (int a = 0; a < 3; ++a) d[a] = pos3[3 * i + a] - (pos3[3 * j + a] + d[a]);
        const double W = orc_W(sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), h);
        sum += m * W;
        one += m / dens[j] * W;
      }
      nd[i] = shepard ? sum / one : sum;
    }
    memcpy(dens, nd, sizeof(double) * (size_t)n);
    free(nd);
  }
  double* pres = (double*)malloc(sizeof(double) * (size_t)n);
  double* snds = (double*)malloc(sizeof(double) * (size_t)n);
  orc_eos(n, dens, pres, snds, cfg->gamma, cfg->rho0, cfg->c0);
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    pair_acc A = {{0, 0, 0}, 0, 0};
    const double poi = pres[i] / (dens[i] * dens[i]);
    for (int k = 0; k < cnts[i]; ++k) {
      const int e = lists[(size_t)i * NB_CAP + k], j = ent_j(e);
      double dr[3], dv[3];
      image_offset(e, cfg, dr);
      for (int a = 0; a < 3; ++a) {
        dr[a] = pos3[3 * i + a] - (pos3[3 * j + a] + dr[a]);
        dv[a] = vel3[3 * i + a] - vel3[3 * j + a];
      }
      pair_term(&cfg->pair, dr, dv, h, h, dens[i], dens[j], poi, pres[j] / (dens[j] * dens[j]), snds[i], snds[j], nu,
                nu, m, &A);
    }
    for (int a = 0; a < 3; ++a) acc3[3 * i + a] = A.acc[a];
    div_v[i] = A.divv / dens[i];
    dt_i[i] = cfg->pair.c_cfl * h / (snds[i] + A.vsig);
  }
  free(pres);
  free(snds);
  free(cnts);
  free(lists);
  table_free(&T);
  free(p4);
}

static void gravity_and_floor(int n, double* acc3, double* dens, const orc_config* cfg) {
  for (int i = 0; i < n; ++i) {
    acc3[3 * i + 2] -= cfg->g;                     /* Dam2.h:104-108 (all particles) */
    dens[i] = fmax(dens[i], cfg->rho_floor);       /* Dam2.h:111 */
  }
}

void orc_initial_force(int n, const double* pos3, const double* vel3, double* dens, double* acc3, double* div_v,
                       double* dt_i, const orc_config* cfg) {
  /* main.cpp:69-78: EoS -> hydro -> (Shepard) -> gravity -> floor.  The
   * summation mode needs its density before the EoS. */
  if (cfg->density_mode == 1) {
    force_pass(n, pos3, vel3, dens, acc3, div_v, dt_i, cfg, 1, 0);
  } else {
    force_pass(n, pos3, vel3, dens, acc3, div_v, dt_i, cfg, 0, 0);
    if (cfg->density_mode == 2) { /* Shepard after the hydro pass (main.cpp:75), FP64 */
      double* a3 = (double*)malloc(sizeof(double) * 3 * (size_t)n);
      double* d1 = (double*)malloc(sizeof(double) * (size_t)n);
      double* t1 = (double*)malloc(sizeof(double) * (size_t)n);
      force_pass(n, pos3, vel3, dens, a3, d1, t1, cfg, 1, 1);
      free(a3);
      free(d1);
      free(t1);
    }
  }
  gravity_and_floor(n, acc3, dens, cfg);
}

double orc_step(int n, double* pos3, double* vel3, double* vel_half3, double* dens, double* acc3, double* div_v,
                double* dt_i, const int32_t* type, const orc_config* cfg, int64_t step_index) {
  const double dt = orc_dt_global(n, acc3, dt_i, type, cfg->h, cfg->nu);
  for (int i = 0; i < n; ++i) { /* class.h:146-159, main.cpp:98-103 */
    if (!type[i])
      for (int a = 0; a < 3; ++a) vel_half3[3 * i + a] = vel3[3 * i + a] + 0.5 * dt * acc3[3 * i + a];
    dens[i] += -dens[i] * dt * div_v[i];
    if (!type[i]) {
      for (int a = 0; a < 3; ++a) {
        pos3[3 * i + a] += dt * vel_half3[3 * i + a];
        vel3[3 * i + a] += dt * acc3[3 * i + a];
      }
    }
    if (cfg->periodic) {
      for (int a = 0; a < 3; ++a) {
        const double L = (double)cfg->hi[a] - (double)cfg->lo[a];
        if (pos3[3 * i + a] >= cfg->hi[a]) pos3[3 * i + a] -= L;
        else if (pos3[3 * i + a] < cfg->lo[a]) pos3[3 * i + a] += L;
      }
    }
  }
  const int do_density = cfg->density_mode == 1 ||
                         (cfg->density_mode == 2 && cfg->shepard_interval > 0 && step_index % cfg->shepard_interval == 0);
  force_pass(n, pos3, vel3, dens, acc3, div_v, dt_i, cfg, do_density, cfg->density_mode == 2);
  gravity_and_floor(n, acc3, dens, cfg);
  for (int i = 0; i < n; ++i) /* class.h:160-163 */
    if (!type[i])
      for (int a = 0; a < 3; ++a) vel3[3 * i + a] = vel_half3[3 * i + a] + 0.5 * dt * acc3[3 * i + a];
  return dt;
}
