/*
 * CPU restatement of XFDTD_CUDA's time-stepping hot path (TEST INFRASTRUCTURE).
 *
 * This file is the oracle of the test-suite: only tests/, the smoke check and
 * the bench's CPU-baseline leg load it, and only as the checker.  The engine
 * never calls it.
 *
 * What it restates, in the reference's own structure and arithmetic order
 * (FP64, every phase a separate sweep over reference-shaped arrays):
 *   step loop        src/domain/domain_hd.cu:35-47
 *                    updateH -> correctH -> updateE -> correctE -> record -> nextStep
 *   Yee update       src/include/updator/update_scheme.cuh:27-63, 141-197
 *                    (eNext/hNext, a==0||b==0 skip for E), 3 component passes
 *                    (basic_updator.cuh:16-32, basic_updator_3d.cu:10-34),
 *                    2-D: Ez only (basic_updator_te.cu:9-20)
 *   ADE update       src/include/updator/ade_updator/template_ade_update_scheme.cuh:17-85,
 *                    src/updator/ade_updator/{debye,drude,m_lor}_ade_updator.cu
 *   CPML corrector   src/boundary/pml_corrector.cu:9-270 (ranges incl. the +1
 *                    tangential extensions and the c==0 shift of the E range)
 *   TFSF corrector   src/include/waveform_source/tfsf/tfsf_corrector.cuh:20-170,
 *                    src/waveform_source/tfsf/tfsf_corrector.cu:18-271 (3-D: 12
 *                    face/component corrections per half step; 2-D: 4)
 *   NF2FF (FD)       src/nf2ff/frequency_domain/nf2ff_frequency_domain.data.cu:80-232,
 *                    src/include/nf2ff/interpolate_scheme.cuh:11-134
 *   NF2FF (TD)       src/nf2ff/time_domain/nf2ff_time_domain_data.cu:113-175,
 *                    src/include/nf2ff/time_domain/nf2ff_time_domain_data.cuh:64-183
 *                    (faces XN..ZP, update<E> then update<H>, :203-223)
 *   movie monitor    src/monitor/movie_monitor.cu:17-46
 * The inputs (coefficients, CPML profiles, TFSF projections, incident tables,
 * NF2FF DFT kernels) are what XFDTD_CORE computes on the host in the
 * reference; here they come from the engine's host scene compiler through
 * xfb_compiled_view, expanded back to the reference's per-cell arrays.
 * The TFSF incident tables e_inc[t][l], h_inc[t][l] are precomputed for all
 * steps, as XFDTD_CORE does, from the 1-D auxiliary recurrence.
 *
 * Parity status: the reference publishes no golden vectors and cannot be
 * compiled here (it needs XFDTD_CORE, xtensor, xtl), so this restatement is
 * "parity unpinned" against reference outputs; it is anchored instead by the
 * analytic known-answer tests in tests/test_oracle_physics.py.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off, so no FMA contraction).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/xfdtd_b200.h"

typedef struct {
  int n0, n1, n2;
  double* d;
} arr3;

static arr3 arr_new(int n0, int n1, int n2) {
  arr3 a;
  a.n0 = n0; a.n1 = n1; a.n2 = n2;
  a.d = (double*)calloc((size_t)n0 * n1 * n2, sizeof(double));
  return a;
}
#define AT(a, i, j, k) ((a).d[((size_t)(i) * (a).n1 + (j)) * (a).n2 + (k)])

enum { EX = 0, EY, EZ, HX, HY, HZ };

typedef struct {
  int on, field, lo[3], hi[3], interval;
  long long frames, count;
  double* data;
} movie_t;

typedef struct orc_sim {
  int dim, nx, ny, nz;
  double dt;
  arr3 f[6];
  arr3 cf[18]; /* reference coefficient arrays, shaped like their field */
  /* ADE */
  int ade_kind, P;
  arr3 ceep, cejsum;
  arr3* cj;    /* [P][7] per-cell pole coefficients (shaped like Ex..Ez? one per cell grid) */
  arr3* J;     /* [3][P] */
  arr3* Jp;    /* [3][P] */
  arr3 Ep[3];
  /* CPML */
  int pml[6];
  const double *ae[3], *be[3], *ah[3], *bh[3];
  arr3 psi[6][4]; /* per face: ea, eb, ha, hb (full field shapes) */
  /* TFSF */
  int tf_on, tf[6];
  const double *pi[3], *ph[3];
  double tre[3], trh[3], ca[3], cb[3];
  int nl;
  double* e_inc; /* [nt][nl+1] */
  double* h_inc; /* [nt][nl]   */
  /* NF2FF */
  int nf_on, nf[6], nfreq;
  const double *te, *th;
  double* acc[64][6][4]; /* [freq][face][ja jb ma mb] complex, face extent */
  int face_n[6][3];
  /* NF2FF time domain */
  int td_on, td[6];
  double td_dir[3], td_ref, d[3], origin[3];
  long long td_bins;
  double* td_pot[6];          /* W_x W_y W_z U_x U_y U_z, [td_bins] */
  double* td_prev[6][2][2];   /* [face][E, H][a, b], face extent */
  int td_n[6][3];
  /* monitors */
  int n_probes;
  int* probe; /* field, i, j, k */
  double* probe_out;
  int n_movies;
  movie_t* movies;
  long long t, total;
} orc_sim;

static void comp_shape(const orc_sim* s, int f, int sh[3]) {
  sh[0] = s->nx + (f == EY || f == EZ || f == HX);
  sh[1] = s->ny + (f == EX || f == EZ || f == HY);
  sh[2] = s->nz + (f == EX || f == EY || f == HZ);
}

/* tangential axes (a, b) of axis c: X->(Y,Z), Y->(Z,X), Z->(X,Y) */
static int ax_a(int c) { return (c + 1) % 3; }
static int ax_b(int c) { return (c + 2) % 3; }
static void abc_to_ijk(int c, int a, int b, int cc, int* i, int* j, int* k) {
  int v[3];
  v[c] = cc; v[ax_a(c)] = a; v[ax_b(c)] = b;
  *i = v[0]; *j = v[1]; *k = v[2];
}
static void ijk_to_abc(int c, int i, int j, int k, int* a, int* b, int* cc) {
  int v[3] = {i, j, k};
  *cc = v[c]; *a = v[ax_a(c)]; *b = v[ax_b(c)];
}

/* coefficient slot of (field c, derivative of dual component d) */
static int coef_index(int attr_h, int comp, int dual) {
  /* E: cexe cexhy cexhz | ceye ceyhz ceyhx | ceze cezhx cezhy
     H: chxh chxey chxez | chyh chyez chyex | chzh chzex chzey */
  int base = (attr_h ? 9 : 0) + 3 * comp;
  if (dual == ax_a(comp)) return base + 1;
  return base + 2;
}

/* Sample point (i, j, k) of `face` (indices inside the face extent) of the
 * time-domain box: the face node along the normal, cell centres along the
 * tangential axes (rVector, nf2ff_time_domain_data.cu:53-66). */
static void td_position(const orc_sim* s, int face, int i, int j, int k, double r[3]) {
  const int c = face / 2, pos = face % 2;
  const int n[3] = {s->td[0] + i + (c == 0 && pos ? s->td[1] - s->td[0] : 0),
                    s->td[2] + j + (c == 1 && pos ? s->td[3] - s->td[2] : 0),
                    s->td[4] + k + (c == 2 && pos ? s->td[5] - s->td[4] : 0)};
  for (int a = 0; a < 3; ++a) r[a] = s->origin[a] + (n[a] + (a == c ? 0.0 : 0.5)) * s->d[a];
}

orc_sim* orc_create(const xfb_compiled_view* v, int n_probes, const int* probes, int n_movies, const int* movies) {
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  s->dim = v->dim; s->nx = v->nx; s->ny = v->ny; s->nz = v->nz; s->dt = v->dt;
  s->total = v->total_steps;
  for (int f = 0; f < 6; ++f) {
    int sh[3];
    comp_shape(s, f, sh);
    s->f[f] = arr_new(sh[0], sh[1], sh[2]);
  }
  /* expand the LUT into per-cell arrays (cell (i,j,k) material for index
     (i,j,k); indices beyond the cells take material 0 and are never used) */
  for (int q = 0; q < 18; ++q) {
    int sh[3];
    comp_shape(s, q < 9 ? q / 3 : 3 + (q - 9) / 3, sh);
    s->cf[q] = arr_new(sh[0], sh[1], sh[2]);
    for (int i = 0; i < sh[0]; ++i)
      for (int j = 0; j < sh[1]; ++j)
        for (int k = 0; k < sh[2]; ++k) {
          int m = 0;
          if (i < s->nx && j < s->ny && k < s->nz) m = v->material_id[((size_t)i * s->ny + j) * s->nz + k];
          AT(s->cf[q], i, j, k) = v->coeff[m * 18 + q];
        }
  }
  s->ade_kind = v->ade_kind;
  s->P = v->ade_poles;
  if (s->ade_kind != XFB_ADE_NONE) {
    const int P = s->P;
    s->ceep = arr_new(s->nx, s->ny, s->nz);
    s->cejsum = arr_new(s->nx, s->ny, s->nz);
    s->cj = (arr3*)calloc((size_t)P * 7, sizeof(arr3));
    s->J = (arr3*)calloc((size_t)3 * P, sizeof(arr3));
    s->Jp = (arr3*)calloc((size_t)3 * P, sizeof(arr3));
    for (int q = 0; q < P * 7; ++q) s->cj[q] = arr_new(s->nx, s->ny, s->nz);
    for (int q = 0; q < 3 * P; ++q) { s->J[q] = arr_new(s->nx, s->ny, s->nz); s->Jp[q] = arr_new(s->nx, s->ny, s->nz); }
    for (int c = 0; c < 3; ++c) s->Ep[c] = arr_new(s->nx, s->ny, s->nz);
    for (int i = 0; i < s->nx; ++i)
      for (int j = 0; j < s->ny; ++j)
        for (int k = 0; k < s->nz; ++k) {
          int m = v->material_id[((size_t)i * s->ny + j) * s->nz + k];
          AT(s->ceep, i, j, k) = v->ade_mat[m * 3 + 1];
          AT(s->cejsum, i, j, k) = v->ade_mat[m * 3 + 2];
          for (int p = 0; p < P; ++p)
            for (int q = 0; q < 7; ++q) AT(s->cj[p * 7 + q], i, j, k) = v->ade_pole[((size_t)m * P + p) * 7 + q];
        }
  }
  for (int q = 0; q < 6; ++q) s->pml[q] = v->pml_cells[q];
  for (int a = 0; a < 3; ++a) { s->ae[a] = v->pml_ae[a]; s->be[a] = v->pml_be[a]; s->ah[a] = v->pml_ah[a]; s->bh[a] = v->pml_bh[a]; }
  for (int face = 0; face < 6; ++face) {
    if (!s->pml[face]) continue;
    const int c = face / 2;
    const int fa = 3 + 0, fb = 0; (void)fa; (void)fb;
    const int ea = ax_a(c), eb = ax_b(c);
    int sh[3];
    comp_shape(s, ea, sh); s->psi[face][0] = arr_new(sh[0], sh[1], sh[2]);
    comp_shape(s, eb, sh); s->psi[face][1] = arr_new(sh[0], sh[1], sh[2]);
    comp_shape(s, 3 + ea, sh); s->psi[face][2] = arr_new(sh[0], sh[1], sh[2]);
    comp_shape(s, 3 + eb, sh); s->psi[face][3] = arr_new(sh[0], sh[1], sh[2]);
  }
  s->tf_on = v->tfsf_enabled;
  if (s->tf_on) {
    memcpy(s->tf, v->tfsf_box, sizeof(s->tf));
    for (int a = 0; a < 3; ++a) {
      s->pi[a] = v->tfsf_proj_int[a]; s->ph[a] = v->tfsf_proj_half[a];
      s->tre[a] = v->tfsf_transform_e[a]; s->trh[a] = v->tfsf_transform_h[a];
      s->ca[a] = v->tfsf_ca[a]; s->cb[a] = v->tfsf_cb[a];
    }
    /* incident tables: row t of e_inc is E_aux at t*dt, row t of h_inc is
       H_aux at (t+1/2)*dt (the tables XFDTD_CORE hands to TFSFCorrectorHD,
       tfsf_corrector_hd.cu:15-22) */
    const int nl = v->aux_nl;
    s->nl = nl;
    const long long nt = v->total_steps > 0 ? v->total_steps : 1;
    s->e_inc = (double*)calloc((size_t)nt * (nl + 1), sizeof(double));
    s->h_inc = (double*)calloc((size_t)nt * nl, sizeof(double));
    double* e = (double*)calloc(nl + 1, sizeof(double));
    double* h = (double*)calloc(nl, sizeof(double));
    for (long long t = 0; t < v->total_steps; ++t) {
      memcpy(s->e_inc + t * (nl + 1), e, (nl + 1) * sizeof(double));
      double e_nlm1 = e[nl - 1], e_nl = e[nl];
      for (int l = 0; l < nl; ++l) h[l] = h[l] + v->aux_chie * (e[l + 1] - e[l]);
      memcpy(s->h_inc + t * nl, h, nl * sizeof(double));
      for (int l = 1; l < nl; ++l) e[l] = e[l] + v->aux_ceih * (h[l] - h[l - 1]);
      e[0] = v->aux_source[t + 1];
      e[nl] = e_nlm1 + v->aux_abc * (e[nl - 1] - e_nl);
    }
    free(e); free(h);
  }
  s->nf_on = v->nf2ff_enabled;
  if (s->nf_on) {
    memcpy(s->nf, v->nf2ff_box, sizeof(s->nf));
    s->nfreq = v->n_freqs;
    s->te = v->nf2ff_te; s->th = v->nf2ff_th;
    for (int face = 0; face < 6; ++face) {
      int n[3] = {s->nf[1] - s->nf[0], s->nf[3] - s->nf[2], s->nf[5] - s->nf[4]};
      n[face / 2] = 1;
      memcpy(s->face_n[face], n, sizeof(n));
      for (int fq = 0; fq < s->nfreq && fq < 64; ++fq)
        for (int w = 0; w < 4; ++w) s->acc[fq][face][w] = (double*)calloc((size_t)2 * n[0] * n[1] * n[2], sizeof(double));
    }
  }
  s->td_on = v->nf2ff_td_enabled;
  s->d[0] = v->dx; s->d[1] = v->dy; s->d[2] = v->dz;
  memcpy(s->origin, v->origin, sizeof(s->origin));
  if (s->td_on) {
    memcpy(s->td, v->nf2ff_td_box, sizeof(s->td));
    s->td_dir[0] = sin(v->nf2ff_td_theta) * cos(v->nf2ff_td_phi);
    s->td_dir[1] = sin(v->nf2ff_td_theta) * sin(v->nf2ff_td_phi);
    s->td_dir[2] = cos(v->nf2ff_td_theta);
    s->td_bins = v->nf2ff_td_bins;
    for (int q = 0; q < 6; ++q) s->td_pot[q] = (double*)calloc((size_t)(s->td_bins > 0 ? s->td_bins : 1), sizeof(double));
    /* reference distance: the largest r . dir over the sample points */
    s->td_ref = -INFINITY;
    for (int face = 0; face < 6; ++face) {
      int n[3] = {s->td[1] - s->td[0], s->td[3] - s->td[2], s->td[5] - s->td[4]};
      n[face / 2] = 1;
      memcpy(s->td_n[face], n, sizeof(n));
      for (int kind = 0; kind < 2; ++kind)
        for (int w = 0; w < 2; ++w) s->td_prev[face][kind][w] = (double*)calloc((size_t)n[0] * n[1] * n[2], sizeof(double));
      for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
          for (int k = 0; k < n[2]; ++k) {
            double r[3];
            td_position(s, face, i, j, k, r);
            const double rd = r[0] * s->td_dir[0] + r[1] * s->td_dir[1] + r[2] * s->td_dir[2];
            if (rd > s->td_ref) s->td_ref = rd;
          }
    }
  }
  s->n_probes = n_probes;
  if (n_probes) {
    s->probe = (int*)malloc(sizeof(int) * 4 * n_probes);
    memcpy(s->probe, probes, sizeof(int) * 4 * n_probes);
    s->probe_out = (double*)calloc((size_t)n_probes * (s->total > 0 ? s->total : 1), sizeof(double));
  }
  s->n_movies = n_movies;
  if (n_movies) {
    s->movies = (movie_t*)calloc(n_movies, sizeof(movie_t));
    for (int m = 0; m < n_movies; ++m) {
      const int* d = movies + 8 * m;
      movie_t* mv = &s->movies[m];
      mv->field = d[0];
      for (int a = 0; a < 3; ++a) { mv->lo[a] = d[1 + a]; mv->hi[a] = d[4 + a]; }
      mv->interval = d[7];
      mv->frames = (s->total + mv->interval - 1) / mv->interval;
      const size_t per = (size_t)(mv->hi[0] - mv->lo[0]) * (mv->hi[1] - mv->lo[1]) * (mv->hi[2] - mv->lo[2]);
      mv->data = (double*)calloc((mv->frames > 0 ? mv->frames : 1) * per, sizeof(double));
    }
  }
  return s;
}

/* ---- Yee updates (update_scheme.cuh:141-197) ----------------------------- */
static inline double e_next(double cece, double ec, double cecha, double ha_p, double ha_q, double cechb, double hb_p,
                            double hb_q) {
  return cece * ec + cecha * (ha_p - ha_q) + cechb * (hb_p - hb_q);
}
static inline double h_next(double chch, double hc, double chcea, double ea_p, double ea_q, double chceb, double eb_p,
                            double eb_q) {
  return chch * hc + chcea * (ea_q - ea_p) + chceb * (eb_q - eb_p);
}

static void update_h(orc_sim* s) {
  for (int c = 0; c < 3; ++c) {
    const int a = ax_a(c), b = ax_b(c);
    arr3* F = &s->f[3 + c];
    const arr3* Fa = &s->f[a];
    const arr3* Fb = &s->f[b];
    const arr3* cc = &s->cf[9 + 3 * c];
    const arr3* ca = &s->cf[9 + 3 * c + 1];
    const arr3* cb = &s->cf[9 + 3 * c + 2];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->nx; ++i)
      for (int j = 0; j < s->ny; ++j)
        for (int k = 0; k < s->nz; ++k) {
          int A, B, C;
          ijk_to_abc(c, i, j, k, &A, &B, &C);
          int ia, ja, ka, ib, jb, kb;
          abc_to_ijk(c, A, B + 1, C, &ia, &ja, &ka);
          abc_to_ijk(c, A + 1, B, C, &ib, &jb, &kb);
          AT(*F, i, j, k) = h_next(AT(*cc, i, j, k), AT(*F, i, j, k), AT(*ca, i, j, k), AT(*Fa, i, j, k),
                                   AT(*Fa, ia, ja, ka), AT(*cb, i, j, k), AT(*Fb, i, j, k), AT(*Fb, ib, jb, kb));
        }
  }
}

static void update_e(orc_sim* s) {
  for (int c = 0; c < 3; ++c) {
    if (s->dim == 2 && c != 2) continue;
    const int a = ax_a(c), b = ax_b(c);
    arr3* F = &s->f[c];
    const arr3* Fa = &s->f[3 + a];
    const arr3* Fb = &s->f[3 + b];
    const arr3* cc = &s->cf[3 * c];
    const arr3* ca = &s->cf[3 * c + 1];
    const arr3* cb = &s->cf[3 * c + 2];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < s->nx; ++i)
      for (int j = 0; j < s->ny; ++j)
        for (int k = 0; k < s->nz; ++k) {
          int A, B, C;
          ijk_to_abc(c, i, j, k, &A, &B, &C);
          if (A == 0 || B == 0) continue;
          int ia, ja, ka, ib, jb, kb;
          abc_to_ijk(c, A, B - 1, C, &ia, &ja, &ka);
          abc_to_ijk(c, A - 1, B, C, &ib, &jb, &kb);
          const double e_cur = AT(*F, i, j, k);
          const double en = e_next(AT(*cc, i, j, k), e_cur, AT(*ca, i, j, k), AT(*Fa, i, j, k), AT(*Fa, ia, ja, ka),
                                   AT(*cb, i, j, k), AT(*Fb, i, j, k), AT(*Fb, ib, jb, kb));
          if (s->ade_kind == XFB_ADE_NONE) {
            AT(*F, i, j, k) = en;
            continue;
          }
          /* TemplateADEUpdateScheme::updateE */
          const int P = s->P;
          double jsum = 0;
          if (s->ade_kind == XFB_ADE_MLORENTZ) {
            for (int p = 0; p < P; ++p)
              jsum += AT(s->cj[p * 7 + 5], i, j, k) * AT(s->J[c * P + p], i, j, k) +
                      AT(s->cj[p * 7 + 6], i, j, k) * AT(s->Jp[c * P + p], i, j, k);
            const double e_prev = AT(s->Ep[c], i, j, k);
            const double e_new = AT(s->ceep, i, j, k) * e_prev + en + AT(s->cejsum, i, j, k) * jsum;
            AT(*F, i, j, k) = e_new;
            for (int p = 0; p < P; ++p) {
              const double jn = AT(s->cj[p * 7 + 2], i, j, k) * e_new + AT(s->cj[p * 7 + 3], i, j, k) * e_cur +
                                AT(s->cj[p * 7 + 4], i, j, k) * e_prev + AT(s->cj[p * 7 + 0], i, j, k) * AT(s->J[c * P + p], i, j, k) +
                                AT(s->cj[p * 7 + 1], i, j, k) * AT(s->Jp[c * P + p], i, j, k);
              AT(s->Jp[c * P + p], i, j, k) = AT(s->J[c * P + p], i, j, k);
              AT(s->J[c * P + p], i, j, k) = jn;
            }
            AT(s->Ep[c], i, j, k) = e_cur;
          } else {
            for (int p = 0; p < P; ++p) jsum += AT(s->cj[p * 7 + 5], i, j, k) * AT(s->J[c * P + p], i, j, k);
            const double e_new = 0.0 * 0.0 + en + AT(s->cejsum, i, j, k) * jsum;
            AT(*F, i, j, k) = e_new;
            for (int p = 0; p < P; ++p) {
              double* jv = &AT(s->J[c * P + p], i, j, k);
              if (s->ade_kind == XFB_ADE_DRUDE)
                *jv = AT(s->cj[p * 7 + 0], i, j, k) * *jv + AT(s->cj[p * 7 + 3], i, j, k) * (e_new + e_cur);
              else
                *jv = AT(s->cj[p * 7 + 0], i, j, k) * *jv + AT(s->cj[p * 7 + 3], i, j, k) * (e_new - e_cur);
            }
          }
        }
  }
}

/* ---- CPML corrector (pml_corrector.cu:9-270) ----------------------------- */
static void correct_pml(orc_sim* s, int face, int attr_h) {
  const int c = face / 2, a = ax_a(c), b = ax_b(c);
  const int n[3] = {s->nx, s->ny, s->nz};
  const int L = s->pml[face];
  if (!L) return;
  const int c0 = (face % 2) ? n[c] - L : 0, c1 = (face % 2) ? n[c] : L;
  const int na = n[a], nb = n[b];
  const int off = (!attr_h && c0 == 0) ? 1 : 0; /* main_axis_offset (c == 0) */
  for (int w = 0; w < 2; ++w) {
    /* w = 0: field of axis a (dual = axis b); w = 1: field of axis b (dual = a) */
    const int comp = w == 0 ? a : b, dual = w == 0 ? b : a;
    int a_end = na, b_end = nb;
    if (!attr_h) { if (w == 0) b_end = nb + 1; else a_end = na + 1; }
    else { if (w == 0) a_end = na + 1; else b_end = nb + 1; }
    arr3* F = &s->f[(attr_h ? 3 : 0) + comp];
    const arr3* D = &s->f[(attr_h ? 0 : 3) + dual];
    arr3* psi = &s->psi[face][(attr_h ? 2 : 0) + w];
    const arr3* cps = &s->cf[coef_index(attr_h, comp, dual)];
    const double* ca = attr_h ? s->ah[c] : s->ae[c];
    const double* cb = attr_h ? s->bh[c] : s->be[c];
#pragma omp parallel for collapse(2) schedule(static)
    for (int cc = c0 + off; cc < c1 + off; ++cc)
      for (int A = 0; A < a_end; ++A)
        for (int B = 0; B < b_end; ++B) {
          int i, j, k, id, jd, kd;
          abc_to_ijk(c, A, B, cc, &i, &j, &k);
          abc_to_ijk(c, A, B, cc + (attr_h ? 1 : -1), &id, &jd, &kd);
          const double dp = AT(*D, i, j, k), dq = AT(*D, id, jd, kd);
          double* pv = &AT(*psi, i, j, k);
          if (!attr_h) *pv = cb[cc] * *pv + ca[cc] * (dp - dq);
          else *pv = cb[cc] * *pv + ca[cc] * (dq - dp);
          AT(*F, i, j, k) += AT(*cps, i, j, k) * *pv;
        }
  }
}

/* ---- TFSF corrector (tfsf_corrector.cuh:20-170, tfsf_corrector.cu:18-130) */
static double lerp_tab(const double* row, double proj) {
  const size_t idx = (size_t)proj;
  const double w = proj - (double)idx;
  return (1 - w) * row[idx] + w * row[idx + 1];
}
static double get_inc(const orc_sim* s, int attr_h, int comp, long long t, int i, int j, int k) {
  const int is = s->tf[0], js = s->tf[2], ks = s->tf[4];
  double p;
  if (!attr_h) {
    if (comp == 0) p = s->ph[0][i - is + 1] + s->pi[1][j - js] + s->pi[2][k - ks];
    else if (comp == 1) p = s->pi[0][i - is] + s->ph[1][j - js + 1] + s->pi[2][k - ks];
    else p = s->pi[0][i - is] + s->pi[1][j - js] + s->ph[2][k - ks + 1];
    return s->tre[comp] * lerp_tab(s->e_inc + t * (s->nl + 1), p);
  }
  if (comp == 0) p = s->pi[0][i - is] + s->ph[1][j - js + 1] + s->ph[2][k - ks + 1] - 0.5;
  else if (comp == 1) p = s->ph[0][i - is + 1] + s->pi[1][j - js] + s->ph[2][k - ks + 1] - 0.5;
  else p = s->ph[0][i - is + 1] + s->ph[1][j - js + 1] + s->pi[2][k - ks] - 0.5;
  return s->trh[comp] * lerp_tab(s->h_inc + t * s->nl, p);
}

/* one correctTFSF<direction, attribute, field_xyz> launch over its whole face */
static void correct_tfsf(orc_sim* s, int face, int attr_h, int fxyz) {
  const int c = face / 2, neg = (face % 2) == 0;
  const int a = ax_a(c), b = ax_b(c);
  const int lo[3] = {s->tf[0], s->tf[2], s->tf[4]}, hi[3] = {s->tf[1], s->tf[3], s->tf[5]};
  int as_ = lo[a], ae_ = hi[a], bs_ = lo[b], be_ = hi[b];
  const int cs = neg ? lo[c] : hi[c];
  const int offset_a = ((!attr_h && fxyz == b) || (attr_h && fxyz == a)) ? 1 : 0;
  if (offset_a) ae_ += 1; else be_ += 1;
  const int dual_field = fxyz == a ? b : a;
  const int equation_flag = attr_h ? -1 : 1;
  const int different_flag = fxyz == a ? -1 : 1;
  const int direction_flag = neg ? -1 : 1;
  const double coef = (attr_h ? s->cb[c] : s->ca[c]) * (equation_flag * different_flag * direction_flag);
  const long long t = s->t;
  arr3* F = &s->f[(attr_h ? 3 : 0) + fxyz];
  for (int A = as_; A < ae_; ++A)
    for (int B = bs_; B < be_; ++B) {
      int i, j, k;
      abc_to_ijk(c, A, B, cs, &i, &j, &k);
      if (neg) {
        if (!attr_h) {
          int id, jd, kd;
          abc_to_ijk(c, A, B, cs - 1, &id, &jd, &kd);
          AT(*F, i, j, k) += get_inc(s, 1, dual_field, t, id, jd, kd) * coef;
        } else {
          int ii, jj, kk;
          abc_to_ijk(c, A, B, cs - 1, &ii, &jj, &kk);
          AT(*F, ii, jj, kk) += get_inc(s, 0, dual_field, t, i, j, k) * coef;
        }
      } else {
        AT(*F, i, j, k) += get_inc(s, attr_h ? 0 : 1, dual_field, t, i, j, k) * coef;
      }
    }
}

static void tfsf_half(orc_sim* s, int attr_h) {
  if (!s->tf_on) return;
  enum { XN = 0, XP, YN, YP, ZN, ZP };
  if (s->dim == 2) { /* TFSFCorrector2DAgency (tfsf_corrector.cu:155-189) */
    if (!attr_h) {
      correct_tfsf(s, XN, 0, 2); correct_tfsf(s, XP, 0, 2); correct_tfsf(s, YN, 0, 2); correct_tfsf(s, YP, 0, 2);
    } else {
      correct_tfsf(s, XN, 1, 1); correct_tfsf(s, XP, 1, 1); correct_tfsf(s, YN, 1, 0); correct_tfsf(s, YP, 1, 0);
    }
    return;
  }
  /* TFSFCorrector3DAgency (tfsf_corrector.cu:201-271) */
  const int order[12][2] = {{XN, 2}, {XP, 2}, {YN, 2}, {YP, 2}, {ZN, 0}, {ZP, 0},
                            {YN, 0}, {YP, 0}, {ZN, 1}, {ZP, 1}, {XN, 1}, {XP, 1}};
  for (int q = 0; q < 12; ++q) correct_tfsf(s, order[q][0], attr_h, order[q][1]);
}

/* ---- NF2FF frequency domain (nf2ff_frequency_domain.data.cu:80-194) ------- */
static double interp(const orc_sim* s, int c, int fld, int i, int j, int k) {
  const arr3* F = &s->f[fld];
#define V(ii, jj, kk) AT(*F, ii, jj, kk)
  if (c == 0) {
    if (fld == EY) return 0.5 * (V(i, j, k + 1) + V(i, j, k));
    if (fld == EZ) return 0.5 * (V(i, j + 1, k) + V(i, j, k));
    if (fld == HY) return 0.25 * (V(i, j + 1, k) + V(i, j, k) + V(i - 1, j + 1, k) + V(i - 1, j, k));
    return 0.25 * (V(i, j, k + 1) + V(i, j, k) + V(i - 1, j, k + 1) + V(i - 1, j, k)); /* HZ */
  }
  if (c == 1) {
    if (fld == EZ) return 0.5 * (V(i + 1, j, k) + V(i, j, k));
    if (fld == EX) return 0.5 * (V(i, j, k + 1) + V(i, j, k));
    if (fld == HZ) return 0.25 * (V(i, j, k + 1) + V(i, j, k) + V(i, j - 1, k + 1) + +V(i, j - 1, k));
    return 0.25 * (V(i + 1, j, k) + V(i, j, k) + V(i + 1, j - 1, k) + V(i, j - 1, k)); /* HX */
  }
  if (fld == EX) return 0.5 * (V(i, j + 1, k) + V(i, j, k));
  if (fld == EY) return 0.5 * (V(i + 1, j, k) + V(i, j, k));
  if (fld == HX) return 0.25 * (V(i + 1, j, k) + V(i, j, k) + V(i, j, k - 1) + V(i + 1, j, k - 1));
  return 0.25 * (V(i, j, k) + V(i, j + 1, k) + V(i, j, k - 1) + V(i, j + 1, k - 1)); /* HY */
#undef V
}

static void nf2ff_update(orc_sim* s) {
  if (!s->nf_on) return;
  const long long t = s->t;
  for (int fq = 0; fq < s->nfreq && fq < 64; ++fq) {
    const double* the = s->te + 2 * ((size_t)fq * s->total + t);
    const double* thh = s->th + 2 * ((size_t)fq * s->total + t);
    for (int face = 0; face < 6; ++face) {
      const int c = face / 2, pos = face % 2, a = ax_a(c), b = ax_b(c);
      const int i0 = c == 0 ? (pos ? s->nf[1] : s->nf[0]) : s->nf[0];
      const int j0 = c == 1 ? (pos ? s->nf[3] : s->nf[2]) : s->nf[2];
      const int k0 = c == 2 ? (pos ? s->nf[5] : s->nf[4]) : s->nf[4];
      const int* n = s->face_n[face];
      const double cja = pos ? -1.0 : 1.0, cjb = pos ? 1.0 : -1.0;
      const double cma = pos ? 1.0 : -1.0, cmb = pos ? -1.0 : 1.0;
      double* ja = s->acc[fq][face][0];
      double* jb = s->acc[fq][face][1];
      double* ma = s->acc[fq][face][2];
      double* mb = s->acc[fq][face][3];
      for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
          for (int k = 0; k < n[2]; ++k) {
            const size_t o = 2 * (((size_t)i * n[1] + j) * n[2] + k);
            const int gi = i0 + i, gj = j0 + j, gk = k0 + k;
            /* calculateJ */
            double v = cja * interp(s, c, 3 + b, gi, gj, gk);
            ja[o] += v * thh[0]; ja[o + 1] += v * thh[1];
            v = cjb * interp(s, c, 3 + a, gi, gj, gk);
            jb[o] += v * thh[0]; jb[o + 1] += v * thh[1];
            /* calculateM */
            v = cma * interp(s, c, b, gi, gj, gk);
            ma[o] += v * the[0]; ma[o + 1] += v * the[1];
            v = cmb * interp(s, c, a, gi, gj, gk);
            mb[o] += v * the[0]; mb[o + 1] += v * the[1];
          }
    }
  }
}

/* ---- NF2FF time domain (nf2ff_time_domain_data.cu:113-175) --------------- */
static void nf2ff_td_update(orc_sim* s) {
  if (!s->td_on) return;
  const long long t = s->t;
  const double c0 = 299792458.0; /* __constant__ C_0, nf2ff_time_domain_data.cu:16 */
  for (int face = 0; face < 6; ++face) {
    const int c = face / 2, pos = face % 2, a = ax_a(c), b = ax_b(c);
    const int* n = s->td_n[face];
    const int i0 = c == 0 && pos ? s->td[1] : s->td[0];
    const int j0 = c == 1 && pos ? s->td[3] : s->td[2];
    const int k0 = c == 2 && pos ? s->td[5] : s->td[4];
    for (int kind = 0; kind < 2; ++kind) { /* update<E> (U), then update<H> (W) */
      const double off = kind ? 0.0 : 0.5;
      double ca = kind ? -1.0 : 1.0, cb = kind ? 1.0 : -1.0;
      if (!pos) { ca *= -1.0; cb *= -1.0; }
      double* pa = s->td_pot[(kind ? 0 : 3) + a];
      double* pb = s->td_pot[(kind ? 0 : 3) + b];
      const int fa = kind ? 3 + a : a, fb = kind ? 3 + b : b;
      double* prev_a = s->td_prev[face][kind][0];
      double* prev_b = s->td_prev[face][kind][1];
      const double ds = s->d[a] * s->d[b];
      for (int i = 0; i < n[0]; ++i)
        for (int j = 0; j < n[1]; ++j)
          for (int k = 0; k < n[2]; ++k) {
            const size_t o = ((size_t)i * n[1] + j) * n[2] + k;
            double r[3];
            td_position(s, face, i, j, k, r);
            const double delay = s->td_ref - (r[0] * s->td_dir[0] + r[1] * s->td_dir[1] + r[2] * s->td_dir[2]);
            const double tsd = delay / (c0 * s->dt);
            const long long nn = (long long)floor(tsd + off + (double)t);
            const double f = tsd + off + (double)t - (double)nn;
            const double av = interp(s, c, fa, i0 + i, j0 + j, k0 + k);
            const double bv = interp(s, c, fb, i0 + i, j0 + j, k0 + k);
            const double da = av - prev_a[o], db = bv - prev_b[o];
            pa[nn] += ca * (1 - f) * ds * db;
            pa[nn + 1] += ca * f * ds * db;
            pb[nn] += cb * (1 - f) * ds * da;
            pb[nn + 1] += cb * f * ds * da;
            prev_a[o] = av;
            prev_b[o] = bv;
          }
    }
  }
}

static void record(orc_sim* s) {
  for (int m = 0; m < s->n_movies; ++m) {
    movie_t* mv = &s->movies[m];
    if (mv->count % mv->interval == 0 && mv->count / mv->interval < mv->frames) {
      const long long fr = mv->count / mv->interval;
      const int n0 = mv->hi[0] - mv->lo[0], n1 = mv->hi[1] - mv->lo[1], n2 = mv->hi[2] - mv->lo[2];
      double* o = mv->data + fr * (long long)n0 * n1 * n2;
      for (int i = 0; i < n0; ++i)
        for (int j = 0; j < n1; ++j)
          for (int k = 0; k < n2; ++k) *o++ = AT(s->f[mv->field], mv->lo[0] + i, mv->lo[1] + j, mv->lo[2] + k);
    }
    mv->count++;
  }
  nf2ff_update(s);
  nf2ff_td_update(s);
  for (int p = 0; p < s->n_probes; ++p) {
    const int* d = s->probe + 4 * p;
    s->probe_out[(size_t)p * s->total + s->t] = AT(s->f[d[0]], d[1], d[2], d[3]);
  }
}

int orc_run(orc_sim* s, long long n) {
  if (s->t + n > s->total) return -1;
  for (long long q = 0; q < n; ++q) {
    update_h(s);
    tfsf_half(s, 1);
    for (int face = 0; face < 6; ++face) correct_pml(s, face, 1);
    update_e(s);
    tfsf_half(s, 0);
    for (int face = 0; face < 6; ++face) correct_pml(s, face, 0);
    record(s);
    s->t++;
  }
  return 0;
}

int orc_field_shape(const orc_sim* s, int f, int sh[3]) {
  comp_shape(s, f, sh);
  return 0;
}
const double* orc_field(const orc_sim* s, int f) { return s->f[f].d; }
double* orc_field_mut(orc_sim* s, int f) { return s->f[f].d; }
const double* orc_probe(const orc_sim* s, int p) { return s->probe_out + (size_t)p * s->total; }
const double* orc_movie(const orc_sim* s, int m) { return s->movies[m].data; }
const double* orc_nf2ff(const orc_sim* s, int fq, int face, int w) { return s->acc[fq][face][w]; }
const double* orc_nf2ff_td(const orc_sim* s, int which) { return s->td_on ? s->td_pot[which] : NULL; }
long long orc_nf2ff_td_bins(const orc_sim* s) { return s->td_on ? s->td_bins : 0; }
long long orc_step(const orc_sim* s) { return s->t; }
const double* orc_e_inc(const orc_sim* s) { return s->e_inc; }
const double* orc_h_inc(const orc_sim* s) { return s->h_inc; }

void orc_destroy(orc_sim* s) {
  if (!s) return;
  for (int f = 0; f < 6; ++f) free(s->f[f].d);
  for (int q = 0; q < 18; ++q) free(s->cf[q].d);
  if (s->ade_kind != XFB_ADE_NONE) {
    free(s->ceep.d); free(s->cejsum.d);
    for (int q = 0; q < s->P * 7; ++q) free(s->cj[q].d);
    for (int q = 0; q < 3 * s->P; ++q) { free(s->J[q].d); free(s->Jp[q].d); }
    for (int c = 0; c < 3; ++c) free(s->Ep[c].d);
    free(s->cj); free(s->J); free(s->Jp);
  }
  for (int face = 0; face < 6; ++face)
    for (int w = 0; w < 4; ++w) free(s->psi[face][w].d);
  free(s->e_inc); free(s->h_inc);
  if (s->nf_on)
    for (int fq = 0; fq < s->nfreq && fq < 64; ++fq)
      for (int face = 0; face < 6; ++face)
        for (int w = 0; w < 4; ++w) free(s->acc[fq][face][w]);
  if (s->td_on) {
    for (int q = 0; q < 6; ++q) free(s->td_pot[q]);
    for (int face = 0; face < 6; ++face)
      for (int kind = 0; kind < 2; ++kind)
        for (int w = 0; w < 2; ++w) free(s->td_prev[face][kind][w]);
  }
  free(s->probe); free(s->probe_out);
  for (int m = 0; m < s->n_movies; ++m) free(s->movies[m].data);
  free(s->movies);
  free(s);
}
