/*
 * pfem2_oracle.c -- FP64 CPU restatement of the reference PFEM2 time step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA library:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it. The product path never links or calls it.
 *
 * Parity status: the reference (andreyypopov/pfem2) has no tests, fixtures
 * or golden vectors, and it cannot be built here (it needs deal.II 9.x).
 * This restatement is therefore pinned only by known-answer tests (shape
 * functions, Gauss rules, mapping inverse, mesh measures) and by the
 * analytic Poiseuille solutions the reference drivers impose; parity with
 * the reference binary itself is unpinned.
 *
 * Algorithm sources (reference file:line):
 *   particles  TurekBenchmark/pfem2particle.cpp:701-918 (seed, check, correct,
 *              move, distribute), :276-507 (point location after a move),
 *              :142-166 (closest vertex), :268-274 (patch ordering);
 *              3D tubePoiseuille3D/pfem2particle.cpp:489-691
 *   FEM        cylinder2D/cylinder2D.cc:385-731 (2D), tubePoiseuille3D/tube.cc:165-715 (3D)
 *   solvers    cylinder2D/cylinder2D.cc:736-779 (BiCGStab + Jacobi / SSOR,
 *              absolute residual tolerance), textbook CG
 *   loads      TurekBenchmark/pfem2particle.cpp:920-970,
 *              tubePoiseuille3D/pfem2particle.cpp:693-737
 *   wall push-back  nacaAirfoil/pfem2particle.cpp:919-952
 *   vorticity  cylinderDyM/pfem2particle.cpp:1000-1050
 *   deal.II pieces restated from their mathematics: FE_Q(1) shape functions,
 *   MappingQ1 (bi/trilinear map and its Newton inverse), QGauss(2),
 *   GeometryInfo::is_inside_unit_cell, GridTools::vertex_to_cell_map and
 *   vertex_to_cell_centers_directions, MatrixTools::apply_boundary_values.
 *
 * Deliberate, documented choices where the reference is unordered or
 * ill-defined:
 *   - particle order inside a cell: the reference iterates an
 *     unordered_multimap; here the order is "stable by the previous storage
 *     order" after every move, with re-seeded particles appended in (i,j,k)
 *     loop order. The removal rule of check_cell_for_empty_parts walks this
 *     order.
 *   - a node with zero projection weight gets velocity 0 (reference: 0/0).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/pfem2.h"

#define MAXV 8
#define MAXD 3

typedef struct {
  int dim, nvc, nfc;
  int nv, nc;
  double* X;   /* nv*dim */
  int* cv;     /* nc*nvc */
  int* fb;     /* nc*nfc */
  int *v2c_ptr, *v2c_cell, *v2c_loc;
  double* v2c_dir; /* unit direction vertex -> cell centre, per incidence */
  int nnz;
  int *rp, *ci, *diag;
  int* inc_slot; /* per incidence k and local vertex b: CSR slot of (v_k, cv[c_k][b]) */
  pfem2_case cs;
  int movement_steps, max_per_part;
  unsigned q[3];
  double* f[PFEM2_N_FIELDS];
  double* corr[3];
  /* eliminated matrices and Dirichlet rhs shifts */
  double *Apred[3], *Kp, *Mc[3];
  double *shift_pred[3], *shift_p;
  unsigned char* isdir[4];
  double* dirval[4];
  /* particles */
  int np, cap;
  int* pc;
  double *pxi, *pu, *px;
  /* stats */
  int n_deleted, n_removed, n_reseeded;
  int iters[7];
  double res[7];
  double time;
  int step;
  int threads;
  int assembled;
} omodel;

/* ------------------------------------------------------------------ */
/* FE_Q(1) on the reference cell, deal.II lexicographic vertex order   */
/* ------------------------------------------------------------------ */
static void shape_values(int dim, const double* xi, double* N) {
  int nvc = 1 << dim;
  for (int v = 0; v < nvc; ++v) {
    double s = 1.0;
    for (int d = 0; d < dim; ++d) s *= ((v >> d) & 1) ? xi[d] : (1.0 - xi[d]);
    N[v] = s;
  }
}

static void shape_grads_ref(int dim, const double* xi, double* dN /* nvc*dim */) {
  int nvc = 1 << dim;
  for (int v = 0; v < nvc; ++v)
    for (int d = 0; d < dim; ++d) {
      double s = ((v >> d) & 1) ? 1.0 : -1.0;
      for (int e = 0; e < dim; ++e)
        if (e != d) s *= ((v >> e) & 1) ? xi[e] : (1.0 - xi[e]);
      dN[v * dim + d] = s;
    }
}

static double det_inv(int dim, const double* J, double* Ji) {
  if (dim == 2) {
    double det = J[0] * J[3] - J[1] * J[2];
    if (Ji) {
      Ji[0] = J[3] / det; Ji[1] = -J[1] / det;
      Ji[2] = -J[2] / det; Ji[3] = J[0] / det;
    }
    return det;
  }
  double a = J[0], b = J[1], c = J[2], d = J[3], e = J[4], f = J[5], g = J[6], h = J[7], i = J[8];
  double A = e * i - f * h, B = -(d * i - f * g), C = d * h - e * g;
  double det = a * A + b * B + c * C;
  if (Ji) {
    Ji[0] = A / det; Ji[1] = -(b * i - c * h) / det; Ji[2] = (b * f - c * e) / det;
    Ji[3] = B / det; Ji[4] = (a * i - c * g) / det;  Ji[5] = -(a * f - c * d) / det;
    Ji[6] = C / det; Ji[7] = -(a * h - b * g) / det; Ji[8] = (a * e - b * d) / det;
  }
  return det;
}

/* x = sum_v N_v(xi) X_v  (MappingQ1::transform_unit_to_real_cell) */
static void map_to_real(const omodel* m, int c, const double* xi, double* x) {
  double N[MAXV];
  shape_values(m->dim, xi, N);
  for (int a = 0; a < m->dim; ++a) x[a] = 0.0;
  for (int v = 0; v < m->nvc; ++v) {
    const double* Xv = m->X + (size_t)m->cv[(size_t)c * m->nvc + v] * m->dim;
    for (int a = 0; a < m->dim; ++a) x[a] += N[v] * Xv[a];
  }
}

/* J[a*dim+b] = dx_a / dxi_b */
static void jacobian(const omodel* m, int c, const double* xi, double* J) {
  double dN[MAXV * MAXD];
  shape_grads_ref(m->dim, xi, dN);
  int dim = m->dim;
  for (int k = 0; k < dim * dim; ++k) J[k] = 0.0;
  for (int v = 0; v < m->nvc; ++v) {
    const double* Xv = m->X + (size_t)m->cv[(size_t)c * m->nvc + v] * dim;
    for (int a = 0; a < dim; ++a)
      for (int b = 0; b < dim; ++b) J[a * dim + b] += Xv[a] * dN[v * dim + b];
  }
}

/* Newton inverse of the multilinear map (MappingQ1::transform_real_to_unit_cell).
 * Returns 0 when the iteration fails, which the reference treats as
 * "not in this cell" (ExcTransformationFailed, TurekBenchmark/pfem2particle.cpp:294-300). */
static int map_to_unit(const omodel* m, int c, const double* x, double* xi) {
  int dim = m->dim;
  for (int d = 0; d < dim; ++d) xi[d] = 0.5;
  for (int it = 0; it < 30; ++it) {
    double F[MAXD], J[9], Ji[9];
    map_to_real(m, c, xi, F);
    jacobian(m, c, xi, J);
    double det = det_inv(dim, J, Ji);
    if (!(det > 0.0)) return 0;
    double dxi[MAXD], mx = 0.0;
    for (int a = 0; a < dim; ++a) {
      double s = 0.0;
      for (int b = 0; b < dim; ++b) s += Ji[a * dim + b] * (F[b] - x[b]);
      dxi[a] = s;
    }
    for (int a = 0; a < dim; ++a) {
      xi[a] -= dxi[a];
      if (fabs(dxi[a]) > mx) mx = fabs(dxi[a]);
      if (!(fabs(xi[a]) < 1e6)) return 0;
    }
    if (mx < 1e-12) return 1;
  }
  return 0;
}

/* GeometryInfo<dim>::is_inside_unit_cell(p): exact [0,1]^dim test. */
static int inside_unit(int dim, const double* xi) {
  for (int d = 0; d < dim; ++d)
    if (!(xi[d] >= 0.0 && xi[d] <= 1.0)) return 0;
  return 1;
}

/* ------------------------------------------------------------------ */
/* QGauss(2) element values                                            */
/* ------------------------------------------------------------------ */
typedef struct {
  double N[MAXV];
  double G[MAXV * MAXD]; /* physical gradients */
  double JxW;
  double n[MAXD];        /* face outward normal (face values only) */
  double x[MAXD];
} qpoint;

static const double GA = 0.21132486540518711775; /* 0.5 - 0.5/sqrt(3) */
static const double GB = 0.78867513459481288225;

static void fill_qpoint(const omodel* m, int c, const double* xi, double w, int face, qpoint* q) {
  int dim = m->dim, nvc = m->nvc;
  double dN[MAXV * MAXD], J[9], Ji[9];
  shape_values(dim, xi, q->N);
  shape_grads_ref(dim, xi, dN);
  jacobian(m, c, xi, J);
  double det = det_inv(dim, J, Ji);
  for (int v = 0; v < nvc; ++v)
    for (int a = 0; a < dim; ++a) {
      double s = 0.0;
      for (int b = 0; b < dim; ++b) s += dN[v * dim + b] * Ji[b * dim + a];
      q->G[v * dim + a] = s;
    }
  map_to_real(m, c, xi, q->x);
  if (face < 0) {
    q->JxW = det * w;
  } else {
    int ax = face / 2;
    double sgn = (face % 2) ? 1.0 : -1.0;
    /* Nanson: n dA = det J J^{-T} N_ref dA_ref */
    double v[MAXD], nn = 0.0;
    for (int a = 0; a < dim; ++a) {
      v[a] = Ji[ax * dim + a] * sgn;
      nn += v[a] * v[a];
    }
    nn = sqrt(nn);
    for (int a = 0; a < dim; ++a) q->n[a] = v[a] / nn;
    q->JxW = det * nn * w;
  }
}

static int cell_qpoints(const omodel* m, int c, qpoint* qs) {
  int dim = m->dim, n = 0;
  double g[2] = {GA, GB};
  if (dim == 2) {
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) {
        double xi[2] = {g[i], g[j]};
        fill_qpoint(m, c, xi, 0.25, -1, &qs[n++]);
      }
  } else {
    for (int k = 0; k < 2; ++k)
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) {
          double xi[3] = {g[i], g[j], g[k]};
          fill_qpoint(m, c, xi, 0.125, -1, &qs[n++]);
        }
  }
  return n;
}

static int face_qpoints(const omodel* m, int c, int f, qpoint* qs) {
  int dim = m->dim, ax = f / 2, n = 0;
  double side = (double)(f % 2);
  double g[2] = {GA, GB};
  if (dim == 2) {
    for (int i = 0; i < 2; ++i) {
      double xi[2];
      xi[ax] = side;
      xi[1 - ax] = g[i];
      fill_qpoint(m, c, xi, 0.5, f, &qs[n++]);
    }
  } else {
    int o1 = (ax == 0) ? 1 : 0, o2 = (ax == 2) ? 1 : 2;
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) {
        double xi[3];
        xi[ax] = side;
        xi[o1] = g[i];
        xi[o2] = g[j];
        fill_qpoint(m, c, xi, 0.25, f, &qs[n++]);
      }
  }
  return n;
}

/* ------------------------------------------------------------------ */
/* model construction                                                  */
/* ------------------------------------------------------------------ */
static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}

static int csr_slot(const omodel* m, int row, int col) {
  int lo = m->rp[row], hi = m->rp[row + 1] - 1;
  while (lo <= hi) {
    int mid = (lo + hi) >> 1;
    if (m->ci[mid] == col) return mid;
    if (m->ci[mid] < col) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

static double bc_value(const pfem2_dirichlet* d, const double* x) {
  if (d->kind == PFEM2_BC_PARABOLA) {
    double s = x[d->axis];
    double L = d->b - d->a;
    return d->value * 4.0 * (s - d->a) * (d->b - s) / (L * L);
  }
  return d->value;
}

static void build_dirichlet(omodel* m, int field) {
  int nvc = m->nvc, dim = m->dim;
  unsigned char* isd = m->isdir[field];
  double* val = m->dirval[field];
  memset(isd, 0, (size_t)m->nv);
  for (int v = 0; v < m->nv; ++v) val[v] = 0.0;
  for (int k = 0; k < m->cs.n_dirichlet[field]; ++k) {
    const pfem2_dirichlet* d = &m->cs.dirichlet[field][k];
    for (int c = 0; c < m->nc; ++c)
      for (int f = 0; f < m->nfc; ++f) {
        if (m->fb[(size_t)c * m->nfc + f] != d->boundary_id) continue;
        int ax = f / 2, side = f % 2;
        for (int v = 0; v < nvc; ++v) {
          if (((v >> ax) & 1) != side) continue;
          int g = m->cv[(size_t)c * nvc + v];
          isd[g] = 1;
          val[g] = bc_value(d, m->X + (size_t)g * dim);
        }
      }
  }
}

static void* xcalloc(size_t n, size_t s) {
  void* p = calloc(n ? n : 1, s);
  if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
  return p;
}

omodel* or_create(int dim, int nv, int nc, const double* X, const int* cells, const int* face_bid,
                  const pfem2_case* cs, int movement_steps, int max_per_part) {
  omodel* m = (omodel*)xcalloc(1, sizeof(omodel));
  m->dim = dim; m->nvc = 1 << dim; m->nfc = 2 * dim;
  m->nv = nv; m->nc = nc;
  m->cs = *cs;
  m->movement_steps = movement_steps;
  m->max_per_part = max_per_part;
  m->threads = 1;
  m->X = (double*)xcalloc((size_t)nv * dim, sizeof(double));
  memcpy(m->X, X, sizeof(double) * nv * dim);
  m->cv = (int*)xcalloc((size_t)nc * m->nvc, sizeof(int));
  memcpy(m->cv, cells, sizeof(int) * (size_t)nc * m->nvc);
  m->fb = (int*)xcalloc((size_t)nc * m->nfc, sizeof(int));
  memcpy(m->fb, face_bid, sizeof(int) * (size_t)nc * m->nfc);

  /* vertex -> cells (GridTools::vertex_to_cell_map: a std::set, ascending cell index) */
  int nvc = m->nvc;
  m->v2c_ptr = (int*)xcalloc((size_t)nv + 1, sizeof(int));
  for (size_t k = 0; k < (size_t)nc * nvc; ++k) m->v2c_ptr[m->cv[k] + 1]++;
  for (int v = 0; v < nv; ++v) m->v2c_ptr[v + 1] += m->v2c_ptr[v];
  int ninc = m->v2c_ptr[nv];
  m->v2c_cell = (int*)xcalloc(ninc, sizeof(int));
  m->v2c_loc = (int*)xcalloc(ninc, sizeof(int));
  m->v2c_dir = (double*)xcalloc((size_t)ninc * dim, sizeof(double));
  int* fill = (int*)xcalloc(nv, sizeof(int));
  for (int c = 0; c < nc; ++c)
    for (int b = 0; b < nvc; ++b) {
      int v = m->cv[(size_t)c * nvc + b];
      int k = m->v2c_ptr[v] + fill[v]++;
      m->v2c_cell[k] = c;
      m->v2c_loc[k] = b;
    }
  free(fill);
  /* direction vertex -> cell centre (vertex average), normalised
   * (GridTools::vertex_to_cell_centers_directions) */
  for (int v = 0; v < nv; ++v)
    for (int k = m->v2c_ptr[v]; k < m->v2c_ptr[v + 1]; ++k) {
      int c = m->v2c_cell[k];
      double ctr[MAXD] = {0, 0, 0}, nn = 0.0;
      for (int b = 0; b < nvc; ++b)
        for (int a = 0; a < dim; ++a) ctr[a] += m->X[(size_t)m->cv[(size_t)c * nvc + b] * dim + a];
      for (int a = 0; a < dim; ++a) {
        ctr[a] = ctr[a] / nvc - m->X[(size_t)v * dim + a];
        nn += ctr[a] * ctr[a];
      }
      nn = sqrt(nn);
      for (int a = 0; a < dim; ++a) m->v2c_dir[(size_t)k * dim + a] = ctr[a] / nn;
    }

  /* CSR sparsity (DoFTools::make_sparsity_pattern for Q1: vertices sharing a cell) */
  m->rp = (int*)xcalloc((size_t)nv + 1, sizeof(int));
  int* tmp = (int*)xcalloc((size_t)nvc * 64, sizeof(int));
  int tmpcap = nvc * 64;
  int** rows = (int**)xcalloc(nv, sizeof(int*));
  int* rlen = (int*)xcalloc(nv, sizeof(int));
  for (int v = 0; v < nv; ++v) {
    int n = 0;
    for (int k = m->v2c_ptr[v]; k < m->v2c_ptr[v + 1]; ++k) {
      int c = m->v2c_cell[k];
      for (int b = 0; b < nvc; ++b) {
        if (n >= tmpcap) { tmpcap *= 2; tmp = (int*)realloc(tmp, sizeof(int) * tmpcap); }
        tmp[n++] = m->cv[(size_t)c * nvc + b];
      }
    }
    qsort(tmp, n, sizeof(int), cmp_int);
    int u = 0;
    for (int i = 0; i < n; ++i)
      if (u == 0 || tmp[i] != tmp[u - 1]) tmp[u++] = tmp[i];
    rows[v] = (int*)xcalloc(u, sizeof(int));
    memcpy(rows[v], tmp, sizeof(int) * u);
    rlen[v] = u;
    m->rp[v + 1] = m->rp[v] + u;
  }
  free(tmp);
  m->nnz = m->rp[nv];
  m->ci = (int*)xcalloc(m->nnz, sizeof(int));
  m->diag = (int*)xcalloc(nv, sizeof(int));
  for (int v = 0; v < nv; ++v) {
    memcpy(m->ci + m->rp[v], rows[v], sizeof(int) * rlen[v]);
    free(rows[v]);
  }
  free(rows);
  free(rlen);
  for (int v = 0; v < nv; ++v) m->diag[v] = csr_slot(m, v, v);
  m->inc_slot = (int*)xcalloc((size_t)ninc * nvc, sizeof(int));
  for (int v = 0; v < nv; ++v)
    for (int k = m->v2c_ptr[v]; k < m->v2c_ptr[v + 1]; ++k) {
      int c = m->v2c_cell[k];
      for (int b = 0; b < nvc; ++b) m->inc_slot[(size_t)k * nvc + b] = csr_slot(m, v, m->cv[(size_t)c * nvc + b]);
    }

  for (int f = 0; f < PFEM2_N_FIELDS; ++f) m->f[f] = (double*)xcalloc(nv, sizeof(double));
  for (int c = 0; c < 3; ++c) {
    m->corr[c] = (double*)xcalloc(nv, sizeof(double));
    m->Apred[c] = (double*)xcalloc(m->nnz, sizeof(double));
    m->Mc[c] = (double*)xcalloc(m->nnz, sizeof(double));
    m->shift_pred[c] = (double*)xcalloc(nv, sizeof(double));
  }
  m->Kp = (double*)xcalloc(m->nnz, sizeof(double));
  m->shift_p = (double*)xcalloc(nv, sizeof(double));
  for (int f = 0; f < 4; ++f) {
    m->isdir[f] = (unsigned char*)xcalloc(nv, 1);
    m->dirval[f] = (double*)xcalloc(nv, sizeof(double));
  }
  for (int c = 0; c < dim; ++c) build_dirichlet(m, c);
  build_dirichlet(m, 3);
  m->step = 1;
  return m;
}

void or_destroy(omodel* m) {
  if (!m) return;
  free(m->X); free(m->cv); free(m->fb);
  free(m->v2c_ptr); free(m->v2c_cell); free(m->v2c_loc); free(m->v2c_dir);
  free(m->rp); free(m->ci); free(m->diag); free(m->inc_slot);
  for (int f = 0; f < PFEM2_N_FIELDS; ++f) free(m->f[f]);
  for (int c = 0; c < 3; ++c) {
    free(m->corr[c]); free(m->Apred[c]); free(m->Mc[c]); free(m->shift_pred[c]);
  }
  free(m->Kp); free(m->shift_p);
  for (int f = 0; f < 4; ++f) { free(m->isdir[f]); free(m->dirval[f]); }
  free(m->pc); free(m->pxi); free(m->pu); free(m->px);
  free(m);
}

void or_set_threads(omodel* m, int t) { m->threads = t < 1 ? 1 : t; }

/* ------------------------------------------------------------------ */
/* particles                                                            */
/* ------------------------------------------------------------------ */
static void reserve(omodel* m, int n) {
  if (n <= m->cap) return;
  int cap = n + n / 2 + 16;
  int dim = m->dim;
  m->pc = (int*)realloc(m->pc, sizeof(int) * cap);
  m->pxi = (double*)realloc(m->pxi, sizeof(double) * cap * dim);
  m->pu = (double*)realloc(m->pu, sizeof(double) * cap * dim);
  m->px = (double*)realloc(m->px, sizeof(double) * cap * dim);
  if (!m->pc || !m->pxi || !m->pu || !m->px) { fprintf(stderr, "oracle: oom\n"); abort(); }
  m->cap = cap;
}

/* counter-based SplitMix64 stream shared with the CUDA library */
static uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double or_uniform(uint64_t seed, uint64_t ordinal, int axis) {
  uint64_t key = seed * 0xD1B54A32D192ED03ULL + ordinal * 4ULL + (uint64_t)axis;
  return (double)(splitmix64(key) >> 11) * (1.0 / 9007199254740992.0);
}

/* interpolate nodal velocity field at xi of cell c, accumulating vertex by
 * vertex as the reference does (TurekBenchmark/pfem2particle.cpp:713-718) */
static void interp_vel(const omodel* m, int c, const double* xi, double* u) {
  double N[MAXV];
  shape_values(m->dim, xi, N);
  for (int d = 0; d < m->dim; ++d) u[d] = 0.0;
  for (int v = 0; v < m->nvc; ++v) {
    int g = m->cv[(size_t)c * m->nvc + v];
    for (int d = 0; d < m->dim; ++d) u[d] = u[d] + N[v] * m->f[PFEM2_FIELD_VX + d][g];
  }
}

static void push_particle(omodel* m, int c, const double* xi, const double* u) {
  reserve(m, m->np + 1);
  int i = m->np++, dim = m->dim;
  m->pc[i] = c;
  for (int d = 0; d < dim; ++d) {
    m->pxi[(size_t)i * dim + d] = xi[d];
    m->pu[(size_t)i * dim + d] = u[d];
  }
  map_to_real(m, c, xi, m->px + (size_t)i * dim);
}

/* seed_particles / seed_particles_into_cell */
void or_seed(omodel* m, const unsigned* q, uint64_t seed, double jitter) {
  int dim = m->dim;
  m->q[0] = q[0]; m->q[1] = q[1]; m->q[2] = dim == 3 ? q[2] : 1;
  unsigned qz = m->q[2];
  uint64_t Q = (uint64_t)q[0] * q[1] * qz;
  double h[3] = {1.0 / q[0], 1.0 / q[1], 1.0 / qz};
  m->np = 0;
  reserve(m, (int)(Q * m->nc));
  for (int c = 0; c < m->nc; ++c)
    for (unsigned i = 0; i < q[0]; ++i)
      for (unsigned j = 0; j < q[1]; ++j)
        for (unsigned k = 0; k < qz; ++k) {
          unsigned idx[3] = {i, j, k};
          uint64_t ord = (uint64_t)c * Q + ((uint64_t)i * q[1] + j) * qz + k;
          double xi[3], u[3];
          for (int d = 0; d < dim; ++d) {
            xi[d] = (idx[d] + 1.0 / 2) * h[d];
            if (jitter != 0.0) xi[d] += jitter * (2.0 * or_uniform(seed, ord, d) - 1.0);
          }
          interp_vel(m, c, xi, u);
          push_particle(m, c, xi, u);
        }
}

/* correct_particles_velocities */
void or_correct(omodel* m) {
  int dim = m->dim, nvc = m->nvc;
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int p = 0; p < m->np; ++p) {
    double N[MAXV];
    int c = m->pc[p];
    shape_values(dim, m->pxi + (size_t)p * dim, N);
    for (int v = 0; v < nvc; ++v) {
      int g = m->cv[(size_t)c * nvc + v];
      for (int d = 0; d < dim; ++d)
        m->pu[(size_t)p * dim + d] = m->pu[(size_t)p * dim + d] +
            N[v] * (m->f[PFEM2_FIELD_VX + d][g] - m->f[PFEM2_FIELD_OLD_VX + d][g]);
    }
  }
}

/* find_closest_vertex_of_cell (TurekBenchmark/pfem2particle.cpp:142-166) */
static int closest_vertex(const omodel* m, int c, const double* xold, const double* uext) {
  int dim = m->dim;
  double un = 0.0, vn[MAXD];
  for (int d = 0; d < dim; ++d) un += uext[d] * uext[d];
  un = sqrt(un);
  for (int d = 0; d < dim; ++d) vn[d] = uext[d] / un;
  double best = 0.0;
  int bv = 0;
  for (int v = 0; v < m->nvc; ++v) {
    const double* Xv = m->X + (size_t)m->cv[(size_t)c * m->nvc + v] * dim;
    double t[MAXD], tn = 0.0, dot = 0.0;
    for (int d = 0; d < dim; ++d) { t[d] = Xv[d] - xold[d]; tn += t[d] * t[d]; }
    tn = sqrt(tn);
    for (int d = 0; d < dim; ++d) dot += vn[d] * (t[d] / tn);
    if (v == 0) best = dot;
    else if (dot > best) { best = dot; bv = v; }
  }
  return bv;
}

/* one particle's relocation after a sub-step (sort_particles_into_subdomains_and_cells).
 * returns new cell or -1 (deleted) */
static int locate(const omodel* m, int c, const double* x, const double* xold, const double* uext, double* xi_out) {
  int dim = m->dim;
  double xi[MAXD];
  if (map_to_unit(m, c, x, xi) && inside_unit(dim, xi)) {
    for (int d = 0; d < dim; ++d) xi_out[d] = xi[d];
    return c;
  }
  int lv = closest_vertex(m, c, xold, uext);
  int gv = m->cv[(size_t)c * m->nvc + lv];
  const double* Xv = m->X + (size_t)gv * dim;
  double vp[MAXD], vpn = 0.0;
  for (int d = 0; d < dim; ++d) { vp[d] = x[d] - Xv[d]; vpn += vp[d] * vp[d]; }
  vpn = sqrt(vpn);
  for (int d = 0; d < dim; ++d) vp[d] /= vpn;
  int k0 = m->v2c_ptr[gv], n = m->v2c_ptr[gv + 1] - k0;
  int perm[64];
  double key[64];
  if (n > 64) n = 64;
  /* std::sort by descending alignment; stable for <= 16 entries (insertion sort) */
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int d = 0; d < dim; ++d) s += m->v2c_dir[(size_t)(k0 + i) * dim + d] * vp[d];
    key[i] = s;
    perm[i] = i;
  }
  for (int i = 1; i < n; ++i) {
    int pi = perm[i];
    double ki = key[pi];
    int j = i - 1;
    while (j >= 0 && ki > key[perm[j]]) { perm[j + 1] = perm[j]; --j; }
    perm[j + 1] = pi;
  }
  for (int i = 0; i < n; ++i) {
    int cc = m->v2c_cell[k0 + perm[i]];
    if (map_to_unit(m, cc, x, xi) && inside_unit(dim, xi)) {
      for (int d = 0; d < dim; ++d) xi_out[d] = xi[d];
      return cc;
    }
  }
  return -1;
}

/* stable counting sort of the particle arrays by cell; drops cell < 0 */
static void sort_by_cell(omodel* m) {
  int dim = m->dim, n = m->np;
  int* cnt = (int*)xcalloc((size_t)m->nc + 1, sizeof(int));
  for (int p = 0; p < n; ++p)
    if (m->pc[p] >= 0) cnt[m->pc[p] + 1]++;
  for (int c = 0; c < m->nc; ++c) cnt[c + 1] += cnt[c];
  int nn = cnt[m->nc];
  int* pc = (int*)xcalloc(nn, sizeof(int));
  double* xi = (double*)xcalloc((size_t)nn * dim, sizeof(double));
  double* u = (double*)xcalloc((size_t)nn * dim, sizeof(double));
  double* x = (double*)xcalloc((size_t)nn * dim, sizeof(double));
  for (int p = 0; p < n; ++p) {
    int c = m->pc[p];
    if (c < 0) continue;
    int o = cnt[c]++;
    pc[o] = c;
    memcpy(xi + (size_t)o * dim, m->pxi + (size_t)p * dim, sizeof(double) * dim);
    memcpy(u + (size_t)o * dim, m->pu + (size_t)p * dim, sizeof(double) * dim);
    memcpy(x + (size_t)o * dim, m->px + (size_t)p * dim, sizeof(double) * dim);
  }
  free(cnt);
  reserve(m, nn);
  memcpy(m->pc, pc, sizeof(int) * nn);
  memcpy(m->pxi, xi, sizeof(double) * nn * dim);
  memcpy(m->pu, u, sizeof(double) * nn * dim);
  memcpy(m->px, x, sizeof(double) * nn * dim);
  m->np = nn;
  free(pc); free(xi); free(u); free(x);
}

/* move_particles without the final check: PARTICLES_MOVEMENT_STEPS forward
 * Euler sub-steps, each followed by point location. */
void or_advect(omodel* m) {
  int dim = m->dim;
  double dts = m->cs.dt / m->movement_steps;
  int deleted = 0;
  for (int s = 0; s < m->movement_steps; ++s) {
#pragma omp parallel for schedule(static) reduction(+ : deleted) num_threads(m->threads)
    for (int p = 0; p < m->np; ++p) {
      int c = m->pc[p];
      if (c < 0) continue;
      double u[MAXD], xold[MAXD], xi[MAXD];
      interp_vel(m, c, m->pxi + (size_t)p * dim, u);
      double* x = m->px + (size_t)p * dim;
      for (int d = 0; d < dim; ++d) {
        xold[d] = x[d];
        x[d] = x[d] + u[d] * dts;
      }
      /* the reference recomputes the old position from the reference
       * coordinates before the closest-vertex search (:145) */
      double xo[MAXD];
      map_to_real(m, c, m->pxi + (size_t)p * dim, xo);
      (void)xold;
      int nc = locate(m, c, x, xo, u, xi);
      if (nc < 0) { m->pc[p] = -1; ++deleted; continue; }
      m->pc[p] = nc;
      for (int d = 0; d < dim; ++d) m->pxi[(size_t)p * dim + d] = xi[d];
    }
  }
  m->n_deleted = deleted;
  sort_by_cell(m);
}

/* check_cell_for_empty_parts for every cell (TurekBenchmark/pfem2particle.cpp:723-772) */
void or_check_empty(omodel* m) {
  int dim = m->dim;
  unsigned q0 = m->q[0], q1 = m->q[1], q2 = dim == 3 ? m->q[2] : 1;
  double h[3] = {1.0 / q0, 1.0 / q1, 1.0 / q2};
  int nb0 = q0 + 1, nb1 = q1 + 1, nb2 = q2 + 1;
  int nb = nb0 * nb1 * nb2;
  int* cnt = (int*)xcalloc(nb, sizeof(int));
  /* output arrays */
  int cap = m->np + m->nc * (int)(q0 * q1 * q2) + 16;
  int* pc = (int*)xcalloc(cap, sizeof(int));
  double* xi = (double*)xcalloc((size_t)cap * dim, sizeof(double));
  double* u = (double*)xcalloc((size_t)cap * dim, sizeof(double));
  double* x = (double*)xcalloc((size_t)cap * dim, sizeof(double));
  int n = 0, removed = 0, reseeded = 0;
  int p = 0;
  for (int c = 0; c < m->nc; ++c) {
    memset(cnt, 0, sizeof(int) * nb);
    for (; p < m->np && m->pc[p] == c; ++p) {
      const double* pxi = m->pxi + (size_t)p * dim;
      unsigned b[3] = {0, 0, 0};
      for (int d = 0; d < dim; ++d) b[d] = (unsigned)(pxi[d] / h[d]);
      int bi = (b[0] * nb1 + b[1]) * nb2 + b[2];
      cnt[bi]++;
      if (cnt[bi] > m->max_per_part) { ++removed; continue; }
      pc[n] = c;
      memcpy(xi + (size_t)n * dim, pxi, sizeof(double) * dim);
      memcpy(u + (size_t)n * dim, m->pu + (size_t)p * dim, sizeof(double) * dim);
      memcpy(x + (size_t)n * dim, m->px + (size_t)p * dim, sizeof(double) * dim);
      ++n;
    }
    for (unsigned i = 0; i < q0; ++i)
      for (unsigned j = 0; j < q1; ++j)
        for (unsigned k = 0; k < q2; ++k) {
          int bi = (i * nb1 + j) * nb2 + k;
          if (cnt[bi]) continue;
          double nxi[3] = {(i + 1.0 / 2) * h[0], (j + 1.0 / 2) * h[1], (k + 1.0 / 2) * h[2]};
          pc[n] = c;
          memcpy(xi + (size_t)n * dim, nxi, sizeof(double) * dim);
          interp_vel(m, c, nxi, u + (size_t)n * dim);
          map_to_real(m, c, nxi, x + (size_t)n * dim);
          ++n;
          ++reseeded;
        }
  }
  free(cnt);
  reserve(m, n);
  memcpy(m->pc, pc, sizeof(int) * n);
  memcpy(m->pxi, xi, sizeof(double) * n * dim);
  memcpy(m->pu, u, sizeof(double) * n * dim);
  memcpy(m->px, x, sizeof(double) * n * dim);
  m->np = n;
  m->n_removed = removed;
  m->n_reseeded = reseeded;
  free(pc); free(xi); free(u); free(x);
}

void or_move(omodel* m) {
  or_advect(m);
  or_check_empty(m);
}

/* distribute_particle_velocities_to_grid */
void or_project(omodel* m) {
  int dim = m->dim, nvc = m->nvc;
  double* w = m->f[PFEM2_FIELD_NODE_WEIGHT];
  double* acc[3];
  for (int d = 0; d < dim; ++d) acc[d] = (double*)xcalloc(m->nv, sizeof(double));
  for (int v = 0; v < m->nv; ++v) w[v] = 0.0;
  for (int p = 0; p < m->np; ++p) {
    int c = m->pc[p];
    double N[MAXV];
    shape_values(dim, m->pxi + (size_t)p * dim, N);
    for (int v = 0; v < nvc; ++v) {
      int g = m->cv[(size_t)c * nvc + v];
      for (int d = 0; d < dim; ++d) acc[d][g] += N[v] * m->pu[(size_t)p * dim + d];
      w[g] += N[v];
    }
  }
  for (int v = 0; v < m->nv; ++v)
    for (int d = 0; d < dim; ++d) m->f[PFEM2_FIELD_VX + d][v] = w[v] != 0.0 ? acc[d][v] / w[v] : 0.0;
  for (int d = 0; d < dim; ++d) free(acc[d]);
  if (m->cs.zero_after_projection_mask && m->cs.wall_pushback) {
    /* wall push-back (nacaAirfoil/pfem2particle.cpp:919-952): for every wall
     * vertex whose projected velocity has a component above 1e-5, every
     * particle of the cells around it loses N_vertex(xi_p) times that
     * velocity; here per particle, over its cell's wall vertices in
     * ascending local order */
    unsigned char* wall = (unsigned char*)xcalloc(m->nv, 1);
    for (int c = 0; c < m->nc; ++c)
      for (int f = 0; f < m->nfc; ++f) {
        int b = m->fb[(size_t)c * m->nfc + f];
        if (b < 0 || b > 31 || !((m->cs.zero_after_projection_mask >> b) & 1u)) continue;
        int ax = f / 2, side = f % 2;
        for (int v = 0; v < nvc; ++v)
          if (((v >> ax) & 1) == side) wall[m->cv[(size_t)c * nvc + v]] = 1;
      }
    for (int p = 0; p < m->np; ++p) {
      int c = m->pc[p];
      double N[MAXV];
      shape_values(dim, m->pxi + (size_t)p * dim, N);
      for (int v = 0; v < nvc; ++v) {
        int g = m->cv[(size_t)c * nvc + v];
        if (!wall[g]) continue;
        int big = 0;
        for (int d = 0; d < dim; ++d) big |= fabs(m->f[PFEM2_FIELD_VX + d][g]) > 1e-5;
        if (!big) continue;
        for (int d = 0; d < dim; ++d) m->pu[(size_t)p * dim + d] -= N[v] * m->f[PFEM2_FIELD_VX + d][g];
      }
    }
    free(wall);
  }
  if (m->cs.zero_after_projection_mask) {
    for (int c = 0; c < m->nc; ++c)
      for (int f = 0; f < m->nfc; ++f) {
        int b = m->fb[(size_t)c * m->nfc + f];
        if (b < 0 || b > 31 || !((m->cs.zero_after_projection_mask >> b) & 1u)) continue;
        int ax = f / 2, side = f % 2;
        for (int v = 0; v < nvc; ++v)
          if (((v >> ax) & 1) == side)
            for (int d = 0; d < dim; ++d) m->f[PFEM2_FIELD_VX + d][m->cv[(size_t)c * nvc + v]] = 0.0;
      }
  }
}

/* calculate_vorticity (cylinderDyM/pfem2particle.cpp:1000-1050), 2D: per
 * cell, at the QGauss(2) points, w = sum_i (dN_i/dx Vy_i - dN_i/dy Vx_i);
 * the cell's sums of N_v w and N_v over its points are added to its vertices
 * in ascending cell order; node value = quotient (0 where the weight is 0).
 * Returns -1 in 3D. */
int or_vorticity(omodel* m) {
  if (m->dim != 2) return -1;
  double* acc = (double*)xcalloc(m->nv, sizeof(double));
  double* wsum = (double*)xcalloc(m->nv, sizeof(double));
  const double* Vx = m->f[PFEM2_FIELD_VX];
  const double* Vy = m->f[PFEM2_FIELD_VY];
  for (int c = 0; c < m->nc; ++c) {
    qpoint qs[8];
    int nq = cell_qpoints(m, c, qs);
    double lv[MAXV] = {0}, lw[MAXV] = {0};
    for (int k = 0; k < nq; ++k) {
      double w = 0.0;
      for (int i = 0; i < 4; ++i) {
        int g = m->cv[(size_t)c * 4 + i];
        w += qs[k].G[i * 2] * Vy[g] - qs[k].G[i * 2 + 1] * Vx[g];
      }
      for (int v = 0; v < 4; ++v) {
        lv[v] += qs[k].N[v] * w;
        lw[v] += qs[k].N[v];
      }
    }
    for (int v = 0; v < 4; ++v) {
      int g = m->cv[(size_t)c * 4 + v];
      acc[g] += lv[v];
      wsum[g] += lw[v];
    }
  }
  for (int v = 0; v < m->nv; ++v) m->f[PFEM2_FIELD_VORTICITY][v] = wsum[v] != 0.0 ? acc[v] / wsum[v] : 0.0;
  free(acc);
  free(wsum);
  return 0;
}

/* ------------------------------------------------------------------ */
/* FEM assembly (element by element into the CSR pattern)               */
/* ------------------------------------------------------------------ */
static int is_open(const omodel* m, int b) {
  return b >= 0 && b < 32 && ((m->cs.open_boundary_mask >> b) & 1u);
}

/* matrices: kind 0 = prediction of component `comp`, 1 = pressure, 2 = mass */
static void assemble_matrix(const omodel* m, int kind, int comp, double* A) {
  int dim = m->dim, nvc = m->nvc;
  double mu = m->cs.mu, rho = m->cs.rho, dt = m->cs.dt;
  memset(A, 0, sizeof(double) * m->nnz);
  qpoint qs[8];
  for (int c = 0; c < m->nc; ++c) {
    int nq = cell_qpoints(m, c, qs);
    double loc[MAXV * MAXV];
    memset(loc, 0, sizeof(loc));
    for (int iq = 0; iq < nq; ++iq) {
      const qpoint* q = &qs[iq];
      for (int i = 0; i < nvc; ++i)
        for (int j = 0; j < nvc; ++j) {
          double val = 0.0;
          if (kind == 0) {
            double s = 0.0;
            for (int d = 0; d < dim; ++d)
              s += (d == comp ? 4.0 / 3.0 : 1.0) * q->G[i * dim + d] * q->G[j * dim + d];
            val = rho * q->N[i] * q->N[j] + mu * dt * s;
          } else if (kind == 1) {
            for (int d = 0; d < dim; ++d) val += q->G[i * dim + d] * q->G[j * dim + d];
          } else {
            val = q->N[i] * q->N[j];
          }
          loc[i * nvc + j] += val * q->JxW;
        }
    }
    for (int i = 0; i < nvc; ++i) {
      int gi = m->cv[(size_t)c * nvc + i];
      for (int j = 0; j < nvc; ++j) {
        int s = csr_slot(m, gi, m->cv[(size_t)c * nvc + j]);
        A[s] += loc[i * nvc + j];
      }
    }
  }
}

/* MatrixTools::apply_boundary_values with column elimination, restated on the
 * fixed CSR pattern. shift[i] = sum_j Aorig(i,j) g_j over Dirichlet columns j
 * for free rows, and Aorig(i,i) g_i for Dirichlet rows. */
static void eliminate(const omodel* m, double* A, const unsigned char* isd, const double* g, double* shift) {
  for (int i = 0; i < m->nv; ++i) {
    double s = 0.0;
    if (isd[i]) {
      s = A[m->diag[i]] * g[i];
    } else {
      for (int k = m->rp[i]; k < m->rp[i + 1]; ++k)
        if (isd[m->ci[k]]) s += A[k] * g[m->ci[k]];
    }
    shift[i] = s;
  }
  for (int i = 0; i < m->nv; ++i)
    for (int k = m->rp[i]; k < m->rp[i + 1]; ++k) {
      int j = m->ci[k];
      if ((isd[i] || isd[j]) && j != i) A[k] = 0.0;
    }
}

static void apply_rhs_bc(const omodel* m, double* rhs, const unsigned char* isd, const double* shift) {
  for (int i = 0; i < m->nv; ++i) rhs[i] = isd[i] ? shift[i] : rhs[i] - shift[i];
}

void or_assemble_matrices(omodel* m) {
  int dim = m->dim;
  double* zero = (double*)xcalloc(m->nv, sizeof(double));
  for (int c = 0; c < dim; ++c) {
    assemble_matrix(m, 0, c, m->Apred[c]);
    eliminate(m, m->Apred[c], m->isdir[c], m->dirval[c], m->shift_pred[c]);
    assemble_matrix(m, 2, c, m->Mc[c]);
    double* sh = (double*)xcalloc(m->nv, sizeof(double));
    eliminate(m, m->Mc[c], m->isdir[c], zero, sh);
    free(sh);
  }
  assemble_matrix(m, 1, 0, m->Kp);
  eliminate(m, m->Kp, m->isdir[3], m->dirval[3], m->shift_p);
  free(zero);
  m->assembled = 1;
}

/* The right-hand sides are assembled cell by cell. Each cell's local vector
 * goes to a per-cell buffer (cells in parallel), and each vertex then sums
 * its cells' entries in ascending cell order (vertices in parallel): the
 * additions of the serial scatter rhs[cv[c][i]] += loc[i] over ascending c,
 * in the same order, so the result does not depend on the thread count. */
static double* cell_buffer(const omodel* m) { return (double*)xcalloc((size_t)m->nc * m->nvc, sizeof(double)); }
static void gather_cells(const omodel* m, const double* lbuf, double* rhs) {
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int v = 0; v < m->nv; ++v) {
    double s = 0.0;
    for (int k = m->v2c_ptr[v]; k < m->v2c_ptr[v + 1]; ++k) s += lbuf[(size_t)m->v2c_cell[k] * m->nvc + m->v2c_loc[k]];
    rhs[v] = s;
  }
}

/* prediction rhs of component comp */
static void rhs_prediction(const omodel* m, int comp, const double* const* old, const double* const* inner, double* rhs) {
  int dim = m->dim, nvc = m->nvc;
  double mu = m->cs.mu, rho = m->cs.rho, dt = m->cs.dt;
  double* lbuf = cell_buffer(m);
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int c = 0; c < m->nc; ++c) {
    qpoint qs[8];
    const int* cvv = m->cv + (size_t)c * nvc;
    double loc[MAXV] = {0};
    int nq = cell_qpoints(m, c, qs);
    for (int iq = 0; iq < nq; ++iq) {
      const qpoint* q = &qs[iq];
      for (int i = 0; i < nvc; ++i)
        for (int j = 0; j < nvc; ++j) {
          double r = rho * q->N[j] * q->N[i] * old[comp][cvv[j]];
          double t = 0.0;
          for (int d = 0; d < dim; ++d) {
            if (d == comp) continue;
            t += (q->G[i * dim + d] * q->G[j * dim + comp] - 2.0 / 3.0 * q->G[i * dim + comp] * q->G[j * dim + d]) *
                 inner[d][cvv[j]];
          }
          loc[i] += (r - mu * dt * t) * q->JxW;
        }
    }
    for (int f = 0; f < m->nfc; ++f) {
      if (!is_open(m, m->fb[(size_t)c * m->nfc + f])) continue;
      qpoint fq[4];
      int nf = face_qpoints(m, c, f, fq);
      for (int iq = 0; iq < nf; ++iq) {
        const qpoint* q = &fq[iq];
        double g[MAXD][MAXD]; /* g[a][b] = d u_a / d x_b of inner field */
        for (int a = 0; a < dim; ++a)
          for (int b = 0; b < dim; ++b) {
            double s = 0.0;
            for (int v = 0; v < nvc; ++v) s += q->G[v * dim + b] * inner[a][cvv[v]];
            g[a][b] = s;
          }
        double T;
        if (dim == 2) {
          /* cylinder2D/cylinder2D.cc:445,521 */
          T = comp == 0 ? (4.0 / 3.0 * g[0][0] - 2.0 / 3.0 * g[1][1]) : (g[0][1] + g[1][0]);
        } else {
          /* tubePoiseuille3D/tube.cc:269,348,427 */
          T = comp == 0 ? (-2.0 * (g[1][1] + g[2][2]) / 3.0) : (comp == 1 ? g[0][1] : g[0][2]);
        }
        for (int i = 0; i < nvc; ++i) loc[i] += mu * dt * q->N[i] * T * q->n[0] * q->JxW;
      }
    }
    for (int i = 0; i < nvc; ++i) lbuf[(size_t)c * nvc + i] = loc[i];
  }
  gather_cells(m, lbuf, rhs);
  free(lbuf);
}

static void rhs_pressure(const omodel* m, const double* const* pred, double* rhs) {
  int dim = m->dim, nvc = m->nvc;
  double rho = m->cs.rho, dt = m->cs.dt, G = m->cs.open_boundary_pressure_flux;
  double* lbuf = cell_buffer(m);
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int c = 0; c < m->nc; ++c) {
    qpoint qs[8];
    const int* cvv = m->cv + (size_t)c * nvc;
    double loc[MAXV] = {0};
    int nq = cell_qpoints(m, c, qs);
    for (int iq = 0; iq < nq; ++iq) {
      const qpoint* q = &qs[iq];
      for (int i = 0; i < nvc; ++i)
        for (int j = 0; j < nvc; ++j) {
          double s = 0.0;
          for (int d = 0; d < dim; ++d) s += pred[d][cvv[j]] * q->G[i * dim + d];
          loc[i] += rho / dt * s * q->N[j] * q->JxW;
        }
    }
    for (int f = 0; f < m->nfc; ++f) {
      if (!is_open(m, m->fb[(size_t)c * m->nfc + f])) continue;
      qpoint fq[4];
      int nf = face_qpoints(m, c, f, fq);
      for (int iq = 0; iq < nf; ++iq) {
        const qpoint* q = &fq[iq];
        double ux = 0.0;
        for (int v = 0; v < nvc; ++v) ux += q->N[v] * pred[0][cvv[v]];
        for (int i = 0; i < nvc; ++i) {
          loc[i] -= rho / dt * q->N[i] * ux * q->n[0] * q->JxW;
          if (G != 0.0) loc[i] += q->N[i] * G * q->n[0] * q->JxW;
        }
      }
    }
    for (int i = 0; i < nvc; ++i) lbuf[(size_t)c * nvc + i] = loc[i];
  }
  gather_cells(m, lbuf, rhs);
  free(lbuf);
}

static void rhs_correction(const omodel* m, int comp, const double* p, double* rhs) {
  int dim = m->dim, nvc = m->nvc;
  double rho = m->cs.rho, dt = m->cs.dt;
  double* lbuf = cell_buffer(m);
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int c = 0; c < m->nc; ++c) {
    qpoint qs[8];
    const int* cvv = m->cv + (size_t)c * nvc;
    double loc[MAXV] = {0};
    int nq = cell_qpoints(m, c, qs);
    for (int iq = 0; iq < nq; ++iq) {
      const qpoint* q = &qs[iq];
      for (int i = 0; i < nvc; ++i)
        for (int j = 0; j < nvc; ++j)
          loc[i] -= dt / rho * q->N[i] * q->G[j * dim + comp] * p[cvv[j]] * q->JxW;
    }
    for (int i = 0; i < nvc; ++i) lbuf[(size_t)c * nvc + i] = loc[i];
  }
  gather_cells(m, lbuf, rhs);
  free(lbuf);
}

/* ------------------------------------------------------------------ */
/* Krylov solvers (deal.II SolverCG / SolverBicgstab, absolute tolerance) */
/* ------------------------------------------------------------------ */
static void spmv(const omodel* m, const double* A, const double* x, double* y) {
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int i = 0; i < m->nv; ++i) {
    double s = 0.0;
    for (int k = m->rp[i]; k < m->rp[i + 1]; ++k) s += A[k] * x[m->ci[k]];
    y[i] = s;
  }
}
static double dot(int n, const double* a, const double* b) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
/* the Krylov solvers' dot product: in index order with one thread; with
 * more, chunks of 4096 entries summed in parallel (each in index order) and
 * then in chunk order, so that the result is the same for every thread
 * count above one */
enum { kDotChunk = 4096 };
static double dot_m(const omodel* m, int n, const double* a, const double* b) {
  if (m->threads <= 1) return dot(n, a, b);
  const int nch = (n + kDotChunk - 1) / kDotChunk;
  double* part = (double*)xcalloc(nch > 0 ? nch : 1, sizeof(double));
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int ch = 0; ch < nch; ++ch) {
    const int i1 = (ch + 1) * kDotChunk < n ? (ch + 1) * kDotChunk : n;
    double s = 0.0;
    for (int i = ch * kDotChunk; i < i1; ++i) s += a[i] * b[i];
    part[ch] = s;
  }
  double s = 0.0;
  for (int ch = 0; ch < nch; ++ch) s += part[ch];
  free(part);
  return s;
}

/* precond: 0 = Jacobi, 1 = SSOR (omega 1, symmetric Gauss-Seidel) */
static void precond(const omodel* m, int kind, const double* A, const double* r, double* z) {
  int n = m->nv;
  if (kind == 0) {
#pragma omp parallel for schedule(static) num_threads(m->threads)
    for (int i = 0; i < n; ++i) z[i] = r[i] / A[m->diag[i]];
    return;
  }
  /* symmetric Gauss-Seidel: sequential by construction, as deal.II's
   * PreconditionSSOR */
  for (int i = 0; i < n; ++i) {
    double s = r[i];
    for (int k = m->rp[i]; k < m->diag[i]; ++k) s -= A[k] * z[m->ci[k]];
    z[i] = s / A[m->diag[i]];
  }
  for (int i = 0; i < n; ++i) z[i] *= A[m->diag[i]];
  for (int i = n - 1; i >= 0; --i) {
    double s = z[i];
    for (int k = m->diag[i] + 1; k < m->rp[i + 1]; ++k) s -= A[k] * z[m->ci[k]];
    z[i] = s / A[m->diag[i]];
  }
}

static int solve_cg(const omodel* m, const double* A, double* x, const double* b, int pk, double tol, int maxit, double* res_out) {
  int n = m->nv;
  double *r = xcalloc(n, 8), *z = xcalloc(n, 8), *p = xcalloc(n, 8), *q = xcalloc(n, 8);
  spmv(m, A, x, q);
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int i = 0; i < n; ++i) r[i] = b[i] - q[i];
  double res = sqrt(dot_m(m, n, r, r));
  int it = 0;
  if (res > tol) {
    precond(m, pk, A, r, z);
    memcpy(p, z, sizeof(double) * n);
    double rho = dot_m(m, n, r, z);
    for (it = 1; it <= maxit; ++it) {
      spmv(m, A, p, q);
      double alpha = rho / dot_m(m, n, p, q);
#pragma omp parallel for schedule(static) num_threads(m->threads)
      for (int i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
      res = sqrt(dot_m(m, n, r, r));
      if (res <= tol) break;
      precond(m, pk, A, r, z);
      double rn = dot_m(m, n, r, z);
      double beta = rn / rho;
      rho = rn;
#pragma omp parallel for schedule(static) num_threads(m->threads)
      for (int i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    if (it > maxit) it = maxit;
  }
  free(r); free(z); free(p); free(q);
  *res_out = res;
  return it;
}

static int solve_bicgstab(const omodel* m, const double* A, double* x, const double* b, int pk, double tol, int maxit, double* res_out) {
  int n = m->nv;
  double *r = xcalloc(n, 8), *rb = xcalloc(n, 8), *p = xcalloc(n, 8), *v = xcalloc(n, 8);
  double *y = xcalloc(n, 8), *z = xcalloc(n, 8), *t = xcalloc(n, 8);
  spmv(m, A, x, v);
#pragma omp parallel for schedule(static) num_threads(m->threads)
  for (int i = 0; i < n; ++i) r[i] = b[i] - v[i];
  memset(v, 0, sizeof(double) * n);
  double res = sqrt(dot_m(m, n, r, r));
  int it = 0;
  if (res > tol) {
    memcpy(rb, r, sizeof(double) * n);
    double alpha = 1.0, rho = 1.0, omega = 1.0;
    for (it = 1; it <= maxit; ++it) {
      double rhobar = dot_m(m, n, r, rb);
      double beta = rhobar * alpha / (rho * omega);
      rho = rhobar;
#pragma omp parallel for schedule(static) num_threads(m->threads)
      for (int i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
      precond(m, pk, A, p, y);
      spmv(m, A, y, v);
      alpha = rho / dot_m(m, n, rb, v);
#pragma omp parallel for schedule(static) num_threads(m->threads)
      for (int i = 0; i < n; ++i) r[i] -= alpha * v[i];
      res = sqrt(dot_m(m, n, r, r));
      if (res <= tol) {
#pragma omp parallel for schedule(static) num_threads(m->threads)
        for (int i = 0; i < n; ++i) x[i] += alpha * y[i];
        break;
      }
      precond(m, pk, A, r, z);
      spmv(m, A, z, t);
      omega = dot_m(m, n, t, r) / dot_m(m, n, t, t);
#pragma omp parallel for schedule(static) num_threads(m->threads)
      for (int i = 0; i < n; ++i) {
        x[i] += alpha * y[i] + omega * z[i];
        r[i] -= omega * t[i];
      }
      res = sqrt(dot_m(m, n, r, r));
      if (res <= tol) break;
    }
    if (it > maxit) it = maxit;
  }
  free(r); free(rb); free(p); free(v); free(y); free(z); free(t);
  *res_out = res;
  return it;
}

/* tol: the absolute tolerance; rtol > 0 raises it to rtol |b| (the library's
 * relative stopping rule, pfem2_case.vel_rtol / p_rtol) */
static int solve(omodel* m, int slot, const double* A, double* x, const double* b, int kind, int pk, double tol,
                 double rtol) {
  double res = 0.0;
  if (rtol > 0.0) {
    const double bn = sqrt(dot_m(m, m->nv, b, b));
    if (rtol * bn > tol) tol = rtol * bn;
  }
  int it = kind == PFEM2_SOLVER_CG ? solve_cg(m, A, x, b, pk, tol, m->cs.max_iter, &res)
                                   : solve_bicgstab(m, A, x, b, pk, tol, m->cs.max_iter, &res);
  m->iters[slot] = it;
  m->res[slot] = res;
  return res <= tol ? 0 : 1;
}

/* fem_step / assemble_system (cylinder2D/cylinder2D.cc:385-731). precond_p:
 * 0 Jacobi, 1 SSOR for the pressure solve (the reference uses SSOR). */
int or_fem_step(omodel* m, int precond_p) {
  int dim = m->dim, nv = m->nv, bad = 0;
  if (m->cs.reassemble_every_step || !m->assembled) or_assemble_matrices(m);
  for (int d = 0; d < dim; ++d) memcpy(m->f[PFEM2_FIELD_OLD_VX + d], m->f[PFEM2_FIELD_VX + d], sizeof(double) * nv);
  memcpy(m->f[PFEM2_FIELD_OLD_P], m->f[PFEM2_FIELD_P], sizeof(double) * nv);
  double* rhs = (double*)xcalloc(nv, sizeof(double));
  double* inner[3] = {0, 0, 0};
  const double* old[3];
  for (int d = 0; d < dim; ++d) {
    inner[d] = (double*)xcalloc(nv, sizeof(double));
    old[d] = m->f[PFEM2_FIELD_OLD_VX + d];
  }
  int nouter = m->cs.outer_corrections < 1 ? 1 : m->cs.outer_corrections;
  for (int oc = 0; oc < nouter; ++oc) {
    for (int d = 0; d < dim; ++d) memcpy(inner[d], m->f[PFEM2_FIELD_VX + d], sizeof(double) * nv);
    for (int c = 0; c < dim; ++c) {
      double* pred = m->f[PFEM2_FIELD_PRED_VX + c];
      rhs_prediction(m, c, old, (const double* const*)inner, rhs);
      apply_rhs_bc(m, rhs, m->isdir[c], m->shift_pred[c]);
      for (int i = 0; i < nv; ++i)
        if (m->isdir[c][i]) pred[i] = m->dirval[c][i];
      bad |= solve(m, c, m->Apred[c], pred, rhs, m->cs.vel_solver, 0, m->cs.vel_tol, m->cs.vel_rtol);
    }
    const double* pr[3];
    for (int d = 0; d < dim; ++d) pr[d] = m->f[PFEM2_FIELD_PRED_VX + d];
    rhs_pressure(m, pr, rhs);
    apply_rhs_bc(m, rhs, m->isdir[3], m->shift_p);
    double* P = m->f[PFEM2_FIELD_P];
    for (int i = 0; i < nv; ++i)
      if (m->isdir[3][i]) P[i] = m->dirval[3][i];
    bad |= solve(m, 3, m->Kp, P, rhs, m->cs.p_solver, precond_p, m->cs.p_tol, m->cs.p_rtol);
    for (int c = 0; c < dim; ++c) {
      rhs_correction(m, c, P, rhs);
      for (int i = 0; i < nv; ++i)
        if (m->isdir[c][i]) { rhs[i] = 0.0; m->corr[c][i] = 0.0; }
      bad |= solve(m, 4 + c, m->Mc[c], m->corr[c], rhs, m->cs.vel_solver, 0, m->cs.vel_tol, m->cs.vel_rtol);
      for (int i = 0; i < nv; ++i) m->f[PFEM2_FIELD_VX + c][i] = m->f[PFEM2_FIELD_PRED_VX + c][i] + m->corr[c][i];
    }
    memcpy(m->f[PFEM2_FIELD_OLD_P], P, sizeof(double) * nv);
  }
  free(rhs);
  for (int d = 0; d < dim; ++d) free(inner[d]);
  return bad;
}

/* calculate_loads */
void or_loads(const omodel* m, int patch, double* out) {
  int dim = m->dim, nvc = m->nvc;
  const double *P = m->f[PFEM2_FIELD_P], *Vx = m->f[PFEM2_FIELD_VX], *Vy = m->f[PFEM2_FIELD_VY];
  double Fx_nu = 0, Fx_p = 0, Fy_nu = 0, Fy_p = 0, Fz_p = 0;
  for (int c = 0; c < m->nc; ++c) {
    const int* cvv = m->cv + (size_t)c * nvc;
    for (int f = 0; f < m->nfc; ++f) {
      if (m->fb[(size_t)c * m->nfc + f] != patch) continue;
      qpoint fq[4];
      int nf = face_qpoints(m, c, f, fq);
      for (int iq = 0; iq < nf; ++iq) {
        const qpoint* q = &fq[iq];
        double pq = 0.0, dv = 0.0;
        for (int v = 0; v < nvc; ++v) {
          pq += P[cvv[v]] * q->N[v];
          if (dim == 2)
            dv += (Vx[cvv[v]] * q->n[1] - Vy[cvv[v]] * q->n[0]) *
                  (q->G[v * dim + 0] * q->n[0] + q->G[v * dim + 1] * q->n[1]);
        }
        if (dim == 2) {
          Fx_nu += m->cs.mu * dv * q->n[1] * q->JxW;
          Fx_p -= pq * q->n[0] * q->JxW;
          Fy_nu -= m->cs.mu * dv * q->n[0] * q->JxW;
          Fy_p -= pq * q->n[1] * q->JxW;
        } else {
          Fx_p += pq * q->n[0] * q->JxW;
          Fy_p += pq * q->n[1] * q->JxW;
          Fz_p += pq * q->n[2] * q->JxW;
        }
      }
    }
  }
  /* 2D: pressure difference p(a) - p(b) (TurekBenchmark/pfem2particle.cpp:953-956);
   * 3D: the pressure at the probe, the mean over the listed probe DoFs
   * (tubePoiseuille3D/pfem2particle.cpp:726-731) */
  double dp = 0.0;
  if (dim == 2) {
    if (m->cs.probe_a >= 0) dp += P[m->cs.probe_a];
    if (m->cs.probe_b >= 0) dp -= P[m->cs.probe_b];
  } else {
    int np = 0;
    if (m->cs.probe_a >= 0) { dp += P[m->cs.probe_a]; ++np; }
    if (m->cs.probe_b >= 0) { dp += P[m->cs.probe_b]; ++np; }
    if (np) dp /= np;
  }
  if (dim == 2) {
    double s = m->cs.rho * m->cs.load_umean * m->cs.load_umean * m->cs.load_diam;
    out[0] = 2.0 * Fx_nu / s; out[1] = 2.0 * Fx_p / s;
    out[2] = 2.0 * Fy_nu / s; out[3] = 2.0 * Fy_p / s;
  } else {
    out[0] = Fx_p; out[1] = Fy_p; out[2] = Fz_p; out[3] = 0.0;
  }
  out[4] = dp;
}

/* ------------------------------------------------------------------ */
/* Moving mesh (cylinderDyM)                                           */
/* ------------------------------------------------------------------ */
/* vertices on any boundary face (isBoundaryNode of
 * initialize_moving_mesh_nodes, cylinderDyM/pfem2particle.cpp:1131-1136) */
static unsigned char* boundary_vertices(const omodel* m) {
  unsigned char* b = (unsigned char*)xcalloc(m->nv, 1);
  for (int c = 0; c < m->nc; ++c)
    for (int f = 0; f < m->nfc; ++f) {
      if (m->fb[(size_t)c * m->nfc + f] < 0) continue;
      for (int v = 0; v < m->nvc; ++v)
        if (((v >> (f / 2)) & 1) == f % 2) b[m->cv[(size_t)c * m->nvc + v]] = 1;
    }
  return b;
}

/* direction vertex -> cell centre of every incidence (after the mesh moved) */
static void update_v2c_dir(omodel* m) {
  int dim = m->dim, nvc = m->nvc;
  for (int v = 0; v < m->nv; ++v)
    for (int k = m->v2c_ptr[v]; k < m->v2c_ptr[v + 1]; ++k) {
      int c = m->v2c_cell[k];
      double ctr[MAXD] = {0, 0, 0}, nn = 0.0;
      for (int b = 0; b < nvc; ++b)
        for (int a = 0; a < dim; ++a) ctr[a] += m->X[(size_t)m->cv[(size_t)c * nvc + b] * dim + a];
      for (int a = 0; a < dim; ++a) {
        ctr[a] = ctr[a] / nvc - m->X[(size_t)v * dim + a];
        nn += ctr[a] * ctr[a];
      }
      nn = sqrt(nn);
      for (int a = 0; a < dim; ++a) m->v2c_dir[(size_t)k * dim + a] = ctr[a] / nn;
    }
}

/* problem_of_elasticity (cylinderDyM/cylinderDyM.cc:926-976) and solveU
 * (:886-903): the mesh displacement u (dim components per vertex) from
 *   a(u, v) = sum_q [ lambda d_ci N_a d_cj N_b + mu d_cj N_a d_ci N_b
 *                     + delta_ci,cj mu grad N_a . grad N_b ] JxW,
 * zero right-hand side, u = 0 on the boundary ids of fixed_mask and
 * u = disp on body_id (both components), solved by CG to
 * max(tol, rtol |b|) (the reference uses CG with an incomplete Cholesky
 * preconditioner; Jacobi reaches the same solution). Into
 * f[PFEM2_FIELD_DISP_X + d]. Returns the iteration count (-1: no convergence). */
int or_elasticity(omodel* m, double lambda, double mu, unsigned fixed_mask, int body_id, const double* disp,
                  double tol, double rtol, int maxit, double* res_out) {
  const int dim = m->dim, nvc = m->nvc, nv = m->nv, nnz = m->nnz;
  double* K[MAXD][MAXD];
  for (int a = 0; a < dim; ++a)
    for (int b = 0; b < dim; ++b) K[a][b] = (double*)xcalloc(nnz, sizeof(double));
  qpoint qs[8];
  for (int c = 0; c < m->nc; ++c) {
    int nq = cell_qpoints(m, c, qs);
    for (int iq = 0; iq < nq; ++iq) {
      const qpoint* q = &qs[iq];
      for (int ia = 0; ia < nvc; ++ia) {
        const int va = m->cv[(size_t)c * nvc + ia];
        const double* Ga = q->G + ia * dim;
        for (int ib = 0; ib < nvc; ++ib) {
          const int vb = m->cv[(size_t)c * nvc + ib];
          const double* Gb = q->G + ib * dim;
          const int slot = csr_slot(m, va, vb);
          double gg = 0.0;
          for (int d = 0; d < dim; ++d) gg += Ga[d] * Gb[d];
          for (int ci = 0; ci < dim; ++ci)
            for (int cj = 0; cj < dim; ++cj) {
              double v = lambda * Ga[ci] * Gb[cj] + mu * Ga[cj] * Gb[ci];
              if (ci == cj) v += mu * gg;
              K[ci][cj][slot] += v * q->JxW;
            }
        }
      }
    }
  }
  /* constrained vertices and their values */
  unsigned char* fix = (unsigned char*)xcalloc(nv, 1);
  double* g = (double*)xcalloc((size_t)nv * dim, sizeof(double));
  for (int c = 0; c < m->nc; ++c)
    for (int f = 0; f < m->nfc; ++f) {
      int bid = m->fb[(size_t)c * m->nfc + f];
      if (bid < 0) continue;
      int isfix = bid < 32 && ((fixed_mask >> bid) & 1u);
      int isbody = bid == body_id;
      if (!isfix && !isbody) continue;
      for (int v = 0; v < nvc; ++v)
        if (((v >> (f / 2)) & 1) == f % 2) {
          int gv = m->cv[(size_t)c * nvc + v];
          fix[gv] = 1;
          for (int d = 0; d < dim; ++d) g[(size_t)gv * dim + d] = isbody ? disp[d] : 0.0;
        }
    }
  /* symmetric elimination: constrained rows keep their diagonal, the
   * columns of constrained vertices move to the right-hand side */
  double* rhs = (double*)xcalloc((size_t)nv * dim, sizeof(double));
  for (int i = 0; i < nv; ++i)
    for (int k = m->rp[i]; k < m->rp[i + 1]; ++k) {
      int j = m->ci[k];
      for (int a = 0; a < dim; ++a)
        for (int b = 0; b < dim; ++b) {
          if (fix[i]) {
            if (!(j == i && a == b)) K[a][b][k] = 0.0;
          } else if (fix[j]) {
            rhs[(size_t)i * dim + a] -= K[a][b][k] * g[(size_t)j * dim + b];
            K[a][b][k] = 0.0;
          }
        }
    }
  for (int i = 0; i < nv; ++i)
    if (fix[i])
      for (int a = 0; a < dim; ++a) rhs[(size_t)i * dim + a] = K[a][a][m->diag[i]] * g[(size_t)i * dim + a];
  /* CG with Jacobi on the block system (vertex-major vectors) */
  const size_t n = (size_t)nv * dim;
  double *x = (double*)xcalloc(n, sizeof(double)), *r = (double*)xcalloc(n, sizeof(double));
  double *z = (double*)xcalloc(n, sizeof(double)), *p = (double*)xcalloc(n, sizeof(double));
  double *qv = (double*)xcalloc(n, sizeof(double));
  for (int i = 0; i < nv; ++i)
    if (fix[i])
      for (int a = 0; a < dim; ++a) x[(size_t)i * dim + a] = g[(size_t)i * dim + a];
#define OR_KMUL(xx, yy)                                                       \
  for (int i = 0; i < nv; ++i)                                                \
    for (int a = 0; a < dim; ++a) {                                           \
      double s_ = 0.0;                                                        \
      for (int k = m->rp[i]; k < m->rp[i + 1]; ++k)                           \
        for (int b = 0; b < dim; ++b) s_ += K[a][b][k] * (xx)[(size_t)m->ci[k] * dim + b]; \
      (yy)[(size_t)i * dim + a] = s_;                                         \
    }
  OR_KMUL(x, qv);
  for (size_t i = 0; i < n; ++i) r[i] = rhs[i] - qv[i];
  double bn = sqrt(dot((int)n, rhs, rhs));
  if (rtol * bn > tol) tol = rtol * bn;
  double res = sqrt(dot((int)n, r, r));
  int it = 0, ok = res <= tol;
  if (!ok) {
    for (int i = 0; i < nv; ++i)
      for (int a = 0; a < dim; ++a) z[(size_t)i * dim + a] = r[(size_t)i * dim + a] / K[a][a][m->diag[i]];
    memcpy(p, z, sizeof(double) * n);
    double rho = dot((int)n, r, z);
    for (it = 1; it <= maxit; ++it) {
      OR_KMUL(p, qv);
      double alpha = rho / dot((int)n, p, qv);
      for (size_t i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * qv[i]; }
      res = sqrt(dot((int)n, r, r));
      if (res <= tol) { ok = 1; break; }
      for (int i = 0; i < nv; ++i)
        for (int a = 0; a < dim; ++a) z[(size_t)i * dim + a] = r[(size_t)i * dim + a] / K[a][a][m->diag[i]];
      double rn = dot((int)n, r, z);
      double beta = rn / rho;
      rho = rn;
      for (size_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
  }
#undef OR_KMUL
  for (int d = 0; d < dim; ++d)
    for (int i = 0; i < nv; ++i) m->f[PFEM2_FIELD_DISP_X + d][i] = x[(size_t)i * dim + d];
  for (int a = 0; a < dim; ++a)
    for (int b = 0; b < dim; ++b) free(K[a][b]);
  free(fix); free(g); free(rhs); free(x); free(r); free(z); free(p); free(qv);
  if (res_out) *res_out = res;
  return ok ? it : -1;
}

/* is_inside_unit_cell(p, eps) */
static int inside_unit_eps(int dim, const double* xi, double eps) {
  for (int d = 0; d < dim; ++d)
    if (!(xi[d] >= -eps && xi[d] <= 1.0 + eps)) return 0;
  return 1;
}

/* reinterpolate_fields (cylinderDyM/pfem2particle.cpp:1144-1235): every
 * interior vertex takes Vx, Vy(, Vz), P interpolated at its displaced
 * position x + u in the old mesh, searched in the lowest-index cell around
 * it first, then the other cells around it in ascending order (inside with
 * tolerance 1e-5); boundary vertices and vertices found nowhere keep their
 * values. A failed inverse map counts as "not inside" (the reference then
 * tests the previous point, a quirk not reproduced). */
void or_reinterpolate(omodel* m) {
  const int dim = m->dim, nvc = m->nvc, nv = m->nv;
  const int flds[4] = {PFEM2_FIELD_VX, PFEM2_FIELD_VY, dim == 3 ? PFEM2_FIELD_VZ : -1, PFEM2_FIELD_P};
  unsigned char* bnd = boundary_vertices(m);
  double* nw[4];
  for (int k = 0; k < 4; ++k) {
    nw[k] = (double*)xcalloc(nv, sizeof(double));
    if (flds[k] >= 0) memcpy(nw[k], m->f[flds[k]], sizeof(double) * nv);
  }
  for (int v = 0; v < nv; ++v) {
    if (bnd[v] || m->v2c_ptr[v + 1] == m->v2c_ptr[v]) continue;
    double x[MAXD], xi[MAXD];
    for (int d = 0; d < dim; ++d) x[d] = m->X[(size_t)v * dim + d] + m->f[PFEM2_FIELD_DISP_X + d][v];
    int found = -1;
    for (int k = m->v2c_ptr[v]; k < m->v2c_ptr[v + 1] && found < 0; ++k) {
      int c = m->v2c_cell[k];
      if (map_to_unit(m, c, x, xi) && inside_unit_eps(dim, xi, 1e-5)) found = c;
    }
    if (found < 0) continue;
    double N[MAXV];
    shape_values(dim, xi, N);
    for (int k = 0; k < 4; ++k) {
      if (flds[k] < 0) continue;
      double s = 0.0;
      for (int b = 0; b < nvc; ++b) s += N[b] * m->f[flds[k]][m->cv[(size_t)found * nvc + b]];
      nw[k][v] = s;
    }
  }
  for (int k = 0; k < 4; ++k) {
    if (flds[k] >= 0) memcpy(m->f[flds[k]], nw[k], sizeof(double) * nv);
    free(nw[k]);
  }
  free(bnd);
}

/* transform_grid (cylinderDyM/pfem2particle.cpp:1237-1261): every vertex
 * moves by the displacement; then sort_particles_into_subdomains_and_cells
 * (:280-...) on the moved mesh: a particle keeps its physical position, is
 * tried in its cell, else searched in the cells around the cell's vertex
 * closest along the direction it moved relative to the mesh (the reference
 * uses the particle's last advection velocity there); particles found
 * nowhere are deleted. The caller then runs check_empty_cells. */
void or_transform_grid(omodel* m) {
  const int dim = m->dim;
  for (int v = 0; v < m->nv; ++v)
    for (int d = 0; d < dim; ++d) m->X[(size_t)v * dim + d] += m->f[PFEM2_FIELD_DISP_X + d][v];
  update_v2c_dir(m);
  m->assembled = 0;  /* the matrices follow the mesh */
  int deleted = 0;
  for (int p = 0; p < m->np; ++p) {
    int c = m->pc[p];
    if (c < 0) continue;
    double xo[MAXD], uext[MAXD], xi[MAXD];
    const double* x = m->px + (size_t)p * dim;
    map_to_real(m, c, m->pxi + (size_t)p * dim, xo);
    for (int d = 0; d < dim; ++d) uext[d] = x[d] - xo[d];
    int nc = locate(m, c, x, xo, uext, xi);
    if (nc < 0) { m->pc[p] = -1; ++deleted; continue; }
    m->pc[p] = nc;
    for (int d = 0; d < dim; ++d) m->pxi[(size_t)p * dim + d] = xi[d];
  }
  m->n_deleted = deleted;
  sort_by_cell(m);
}

void or_get_vertices(const omodel* m, double* X) { memcpy(X, m->X, sizeof(double) * m->nv * m->dim); }

/* one run() iteration: correct -> move -> distribute -> fem -> time advance */
int or_step(omodel* m, int precond_p) {
  or_correct(m);
  or_move(m);
  or_project(m);
  int bad = or_fem_step(m, precond_p);
  m->time += m->cs.dt;
  m->step += 1;
  return bad;
}

/* ------------------------------------------------------------------ */
/* state access                                                         */
/* ------------------------------------------------------------------ */
int or_n_particles(const omodel* m) { return m->np; }
int or_nnz(const omodel* m) { return m->nnz; }

void or_get_particles(const omodel* m, int* cell, double* xi, double* u) {
  memcpy(cell, m->pc, sizeof(int) * m->np);
  memcpy(xi, m->pxi, sizeof(double) * m->np * m->dim);
  memcpy(u, m->pu, sizeof(double) * m->np * m->dim);
}

void or_get_positions(const omodel* m, double* x) { memcpy(x, m->px, sizeof(double) * m->np * m->dim); }

/* replaces the particles (stable-sorted by cell); physical positions from xi */
void or_set_particles(omodel* m, int n, const int* cell, const double* xi, const double* u, const unsigned* q) {
  int dim = m->dim;
  if (q) { m->q[0] = q[0]; m->q[1] = q[1]; m->q[2] = dim == 3 ? q[2] : 1; }
  m->np = 0;
  reserve(m, n);
  for (int p = 0; p < n; ++p) push_particle(m, cell[p], xi + (size_t)p * dim, u + (size_t)p * dim);
  sort_by_cell(m);
}

void or_get_field(const omodel* m, int f, double* out) { memcpy(out, m->f[f], sizeof(double) * m->nv); }
void or_set_field(omodel* m, int f, const double* in) { memcpy(m->f[f], in, sizeof(double) * m->nv); }

void or_get_stats(const omodel* m, int* ints /*4+7*/, double* res7) {
  ints[0] = m->np; ints[1] = m->n_deleted; ints[2] = m->n_removed; ints[3] = m->n_reseeded;
  for (int k = 0; k < 7; ++k) { ints[4 + k] = m->iters[k]; res7[k] = m->res[k]; }
}

/* matrices for tests: which 0..2 pred, 3 pressure, 4..6 mass; returns nnz */
int or_get_matrix(omodel* m, int which, int* rp, int* ci, double* val) {
  const double* A = which < 3 ? m->Apred[which] : (which == 3 ? m->Kp : m->Mc[which - 4]);
  if (rp) memcpy(rp, m->rp, sizeof(int) * (m->nv + 1));
  if (ci) memcpy(ci, m->ci, sizeof(int) * m->nnz);
  if (val) memcpy(val, A, sizeof(double) * m->nnz);
  return m->nnz;
}

/* unassembled / raw helpers for known-answer tests */
void or_shape_values(int dim, const double* xi, double* N) { shape_values(dim, xi, N); }
int or_map_to_unit(const omodel* m, int c, const double* x, double* xi) { return map_to_unit(m, c, x, xi); }
void or_map_to_real(const omodel* m, int c, const double* xi, double* x) { map_to_real(m, c, xi, x); }
/* measure of the mesh by QGauss(2) (area / volume) */
double or_measure(const omodel* m) {
  qpoint qs[8];
  double s = 0.0;
  for (int c = 0; c < m->nc; ++c) {
    int nq = cell_qpoints(m, c, qs);
    for (int i = 0; i < nq; ++i) s += qs[i].JxW;
  }
  return s;
}
/* length / area of the boundary with id b and the integral of n over it */
double or_boundary_measure(const omodel* m, int b, double* nint) {
  double s = 0.0;
  for (int a = 0; a < m->dim; ++a) nint[a] = 0.0;
  for (int c = 0; c < m->nc; ++c)
    for (int f = 0; f < m->nfc; ++f) {
      if (m->fb[(size_t)c * m->nfc + f] != b) continue;
      qpoint fq[4];
      int nf = face_qpoints(m, c, f, fq);
      for (int i = 0; i < nf; ++i) {
        s += fq[i].JxW;
        for (int a = 0; a < m->dim; ++a) nint[a] += fq[i].n[a] * fq[i].JxW;
      }
    }
  return s;
}
/* rhs of one system for tests: 0..2 prediction comp, 3 pressure, 4..6 correction */
void or_rhs(omodel* m, int which, double* out) {
  int dim = m->dim;
  const double* old[3];
  const double* cur[3];
  const double* pr[3];
  for (int d = 0; d < dim; ++d) {
    old[d] = m->f[PFEM2_FIELD_OLD_VX + d];
    cur[d] = m->f[PFEM2_FIELD_VX + d];
    pr[d] = m->f[PFEM2_FIELD_PRED_VX + d];
  }
  if (which < 3) {
    rhs_prediction(m, which, old, cur, out);
    apply_rhs_bc(m, out, m->isdir[which], m->shift_pred[which]);
  } else if (which == 3) {
    rhs_pressure(m, pr, out);
    apply_rhs_bc(m, out, m->isdir[3], m->shift_p);
  } else {
    rhs_correction(m, which - 4, m->f[PFEM2_FIELD_P], out);
    for (int i = 0; i < m->nv; ++i)
      if (m->isdir[which - 4][i]) out[i] = 0.0;
  }
}
void or_get_dirichlet(const omodel* m, int field, unsigned char* isd, double* val) {
  memcpy(isd, m->isdir[field], m->nv);
  memcpy(val, m->dirval[field], sizeof(double) * m->nv);
}
