/*
 * CPU oracle for the SPH step of Blackhole-Nebula-Simulator.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C (OpenMP) restatement of the reference's
 * per-particle CPU kernels.  It is the checker the CUDA path is compared against, and the CPU
 * baseline timed beside it; nothing in the product path links or calls it.  Every function cites
 * the reference file:line whose algorithm it restates (paths inside the reference project).
 *
 * Conventions follow the reference: float64 C-order (N, 3) positions, int64 CSR neighbour lists
 * whose rows are sorted and include the particle itself, "rows" subsets whose results come back
 * in rows order, and per-row loops that write only their own row (so any thread count gives the
 * same bits).  Arithmetic is written in the reference's operation order and built with
 * -ffp-contract=off so no multiply-add is fused.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define R_KERN 2.0

/* ------------------------------------------------------------------ kernel shapes
 * sim/kernels_nb.py:16-43 (cubic spline kid 0, Wendland C4 kid 1). */
static inline double kernel_f(double q, int kid) {
  if (q >= 2.0) return 0.0;
  if (kid == 0) {
    if (q < 1.0) return 1.0 - 1.5 * q * q + 0.75 * q * q * q;
    double t = 2.0 - q;
    return 0.25 * t * t * t;
  }
  double x = 1.0 - 0.5 * q;
  double x2 = x * x;
  return x2 * x2 * x2 * (35.0 / 12.0 * q * q + 3.0 * q + 1.0);
}

static inline double kernel_df(double q, int kid) {
  if (q >= 2.0) return 0.0;
  if (kid == 0) {
    if (q < 1.0) return -3.0 * q + 2.25 * q * q;
    double t = 2.0 - q;
    return -0.75 * t * t;
  }
  double x = 1.0 - 0.5 * q;
  double x2 = x * x;
  return -7.0 / 3.0 * q * x2 * x2 * x * (5.0 * q + 2.0);
}

double or_kernel_f(double q, int kid) { return kernel_f(q, kid); }
double or_kernel_df(double q, int kid) { return kernel_df(q, kid); }

/* Python's floor-mod for int64 (non-negative for a positive divisor). */
static inline int64_t pymod(int64_t a, int64_t n) {
  int64_t r = a % n;
  return r < 0 ? r + n : r;
}

/* ------------------------------------------------------------------ cell grid
 * sim/neighbours.py:96-126 (_cell_of, _build_grid): x-major cell index (cx*ny+cy)*nz+cz and a
 * stable counting sort (order lists particles cell by cell, ascending index inside a cell). */
static inline int64_t cell_of(double x, double lo, double inv, int64_t nc) {
  int64_t k = (int64_t)floor((x - lo) * inv);
  if (k < 0) k = 0;
  if (k >= nc) k = nc - 1;
  return k;
}

void or_build_grid(int64_t n, const double* pos, const double* lo, const double* inv_cell,
                   const int64_t* ncell, int64_t* cell, int64_t* start, int64_t* order) {
  int64_t total = ncell[0] * ncell[1] * ncell[2];
  for (int64_t i = 0; i < n; ++i) {
    int64_t cx = cell_of(pos[3 * i + 0], lo[0], inv_cell[0], ncell[0]);
    int64_t cy = cell_of(pos[3 * i + 1], lo[1], inv_cell[1], ncell[1]);
    int64_t cz = cell_of(pos[3 * i + 2], lo[2], inv_cell[2], ncell[2]);
    cell[i] = (cx * ncell[1] + cy) * ncell[2] + cz;
  }
  memset(start, 0, sizeof(int64_t) * (size_t)(total + 1));
  for (int64_t i = 0; i < n; ++i) start[cell[i] + 1] += 1;
  for (int64_t c = 0; c < total; ++c) start[c + 1] += start[c];
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total > 0 ? total : 1));
  memcpy(fill, start, sizeof(int64_t) * (size_t)total);
  for (int64_t i = 0; i < n; ++i) order[fill[cell[i]]++] = i;
  free(fill);
}

/* sim/neighbours.py:129-145 (_cell_range). */
static inline void cell_range(double xc, double r, double lo, double inv, int64_t nc,
                              int periodic, int64_t* first, int64_t* count, int* whole) {
  int64_t a = (int64_t)floor((xc - r - lo) * inv);
  int64_t b = (int64_t)floor((xc + r - lo) * inv);
  *whole = 0;
  if (periodic) {
    int64_t cnt = b - a + 1;
    if (cnt >= nc) {
      *first = a;
      *count = nc;
      *whole = 1;
      return;
    }
    *first = a;
    *count = cnt;
    return;
  }
  if (a < 0) a = 0;
  if (b > nc - 1) b = nc - 1;
  *first = a;
  *count = (b - a + 1) > 0 ? (b - a + 1) : 0;
}

/* sim/neighbours.py:148-156 (_image_delta). rint() rounds half to even like np.round. */
static inline double image_delta(double d, double box_c, int64_t raw, int64_t cell, int64_t nc,
                                 int whole) {
  if (box_c <= 0.0) return d;
  if (whole) return d - box_c * rint(d / box_c);
  return d + box_c * (double)((raw - cell) / nc);
}

/* sim/neighbours.py:159-190 (_gather): gather {j : r_ij < 2 h_i}, count pass or fill pass. */
static void gather(int64_t n, const double* pos, const double* h, const double* box,
                   const double* lo, const double* inv, const int64_t* nc, const int64_t* start,
                   const int64_t* order, int64_t* counts, const int64_t* out_off,
                   int64_t* out_idx, int fill_pass) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    double r = R_KERN * h[i];
    double r2 = r * r;
    int64_t m = 0;
    int64_t ax, nx, ay, ny, az, nz;
    int wx, wy, wz;
    cell_range(pos[3 * i + 0], r, lo[0], inv[0], nc[0], box[0] > 0, &ax, &nx, &wx);
    cell_range(pos[3 * i + 1], r, lo[1], inv[1], nc[1], box[1] > 0, &ay, &ny, &wy);
    cell_range(pos[3 * i + 2], r, lo[2], inv[2], nc[2], box[2] > 0, &az, &nz, &wz);
    for (int64_t di = 0; di < nx; ++di) {
      int64_t rx = ax + di, cx = pymod(rx, nc[0]);
      for (int64_t dj = 0; dj < ny; ++dj) {
        int64_t ry = ay + dj, cy = pymod(ry, nc[1]);
        for (int64_t dk = 0; dk < nz; ++dk) {
          int64_t rz = az + dk, cz = pymod(rz, nc[2]);
          int64_t c = (cx * nc[1] + cy) * nc[2] + cz;
          for (int64_t k = start[c]; k < start[c + 1]; ++k) {
            int64_t j = order[k];
            double dx = image_delta(pos[3 * j + 0] - pos[3 * i + 0], box[0], rx, cx, nc[0], wx);
            double dy = image_delta(pos[3 * j + 1] - pos[3 * i + 1], box[1], ry, cy, nc[1], wy);
            double dz = image_delta(pos[3 * j + 2] - pos[3 * i + 2], box[2], rz, cz, nc[2], wz);
            if (dx * dx + dy * dy + dz * dz < r2) {
              if (fill_pass) out_idx[out_off[i] + m] = j;
              m += 1;
            }
          }
        }
      }
    }
    if (!fill_pass) counts[i] = m;
  }
}

static int cmp_i64(const void* a, const void* b) {
  int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
  return (x > y) - (x < y);
}

/* Geometry of the grid exactly as find_neighbours_numba chooses it (sim/neighbours.py:240-265).
 * pos must already be wrapped into the box when periodic. */
static int cmp_f64(const void* a, const void* b) {
  double x = *(const double*)a, y = *(const double*)b;
  return (x > y) - (x < y);
}

void or_grid_geometry(int64_t n, const double* wrapped, const double* h, const double* box,
                      double* lo, double* inv_cell, int64_t* ncell) {
  int periodic = box[0] > 0.0 || box[1] > 0.0 || box[2] > 0.0;
  double span[3];
  if (!periodic) {
    for (int c = 0; c < 3; ++c) {
      double mn = wrapped[c], mx = wrapped[c];
      for (int64_t i = 1; i < n; ++i) {
        double v = wrapped[3 * i + c];
        if (v < mn) mn = v;
        if (v > mx) mx = v;
      }
      lo[c] = mn;
      span[c] = mx - mn;
    }
  } else {
    for (int c = 0; c < 3; ++c) {
      lo[c] = 0.0;
      span[c] = box[c];
    }
  }
  double* hs = (double*)malloc(sizeof(double) * (size_t)n);
  memcpy(hs, h, sizeof(double) * (size_t)n);
  qsort(hs, (size_t)n, sizeof(double), cmp_f64);
  double med = (n % 2) ? hs[n / 2] : (hs[n / 2 - 1] + hs[n / 2]) / 2.0;
  free(hs);
  double smax = span[0];
  if (span[1] > smax) smax = span[1];
  if (span[2] > smax) smax = span[2];
  double cell = 0.5 * R_KERN * med;
  if (smax / 160.0 > cell) cell = smax / 160.0;
  if (1e-300 > cell) cell = 1e-300;
  for (int c = 0; c < 3; ++c) {
    if (periodic) {
      int64_t k = (int64_t)floor(box[c] / cell);
      ncell[c] = k > 1 ? k : 1;
      inv_cell[c] = (double)ncell[c] / box[c];
    } else {
      int64_t k = (int64_t)floor(span[c] / cell) + 1;
      ncell[c] = k > 1 ? k : 1;
      inv_cell[c] = 1.0 / cell;
    }
  }
}

/* sim/neighbours.py:240-281 (find_neighbours_numba): gather lists, rows sorted, transposed and
 * merged into symmetric CSR lists.  Returns the number of entries; *off_out (n+1) and *idx_out
 * are malloc'd here and released with or_free.  box: three lengths, zeros for open. */
int64_t or_find_neighbours(int64_t n, const double* pos_in, const double* h, const double* box,
                           int64_t** off_out, int64_t** idx_out) {
  int periodic = box[0] > 0.0 || box[1] > 0.0 || box[2] > 0.0;
  double* pos = (double*)malloc(sizeof(double) * (size_t)(3 * n + 1));
  for (int64_t i = 0; i < 3 * n; ++i) {
    double v = pos_in[i];
    if (periodic) {
      double b = box[i % 3];
      double r = fmod(v, b);
      if (r != 0.0) {
        if ((b < 0) != (r < 0)) r += b;
      } else {
        r = copysign(0.0, b);
      }
      v = r;
    }
    pos[i] = v;
  }
  double lo[3], inv[3];
  int64_t nc[3];
  or_grid_geometry(n, pos, h, box, lo, inv, nc);
  int64_t total = nc[0] * nc[1] * nc[2];
  int64_t* cell = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  int64_t* start = (int64_t*)malloc(sizeof(int64_t) * (size_t)(total + 1));
  int64_t* order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  or_build_grid(n, pos, lo, inv, nc, cell, start, order);
  int64_t* counts = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  gather(n, pos, h, box, lo, inv, nc, start, order, counts, NULL, NULL, 0);
  int64_t* g_off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  g_off[0] = 0;
  for (int64_t i = 0; i < n; ++i) g_off[i + 1] = g_off[i] + counts[i];
  int64_t* g_idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(g_off[n] + 1));
  gather(n, pos, h, box, lo, inv, nc, start, order, counts, g_off, g_idx, 1);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i)
    qsort(g_idx + g_off[i], (size_t)(g_off[i + 1] - g_off[i]), sizeof(int64_t), cmp_i64);
  /* transpose (sim/neighbours.py:193-207): rows of the transpose come out sorted */
  int64_t m_tot = g_off[n];
  int64_t* t_off = (int64_t*)calloc((size_t)(n + 1), sizeof(int64_t));
  for (int64_t k = 0; k < m_tot; ++k) t_off[g_idx[k] + 1] += 1;
  for (int64_t i = 0; i < n; ++i) t_off[i + 1] += t_off[i];
  int64_t* t_idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m_tot + 1));
  int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  memcpy(fill, t_off, sizeof(int64_t) * (size_t)n);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = g_off[i]; k < g_off[i + 1]; ++k) t_idx[fill[g_idx[k]]++] = i;
  /* merge sorted rows, duplicates removed (sim/neighbours.py:210-231), count then fill */
  int64_t* off = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  for (int pass = 0; pass < 2; ++pass) {
    int64_t* idx = pass ? *idx_out : NULL;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < n; ++i) {
      int64_t p = g_off[i], pe = g_off[i + 1], q = t_off[i], qe = t_off[i + 1];
      int64_t m = 0, last = -1;
      while (p < pe || q < qe) {
        int64_t v;
        if (q >= qe || (p < pe && g_idx[p] <= t_idx[q])) {
          v = g_idx[p++];
        } else {
          v = t_idx[q++];
        }
        if (v != last) {
          if (pass) idx[off[i] + m] = v;
          m += 1;
          last = v;
        }
      }
      if (!pass) counts[i] = m;
    }
    if (!pass) {
      off[0] = 0;
      for (int64_t i = 0; i < n; ++i) off[i + 1] = off[i] + counts[i];
      *idx_out = (int64_t*)malloc(sizeof(int64_t) * (size_t)(off[n] + 1));
    }
  }
  *off_out = off;
  free(pos);
  free(cell);
  free(start);
  free(order);
  free(counts);
  free(g_off);
  free(g_idx);
  free(t_off);
  free(t_idx);
  free(fill);
  return off[n];
}

/* Cell index and (start, order) of the reference grid for given positions and h: the cell
 * assignment the GPU grid is checked against (sim/neighbours.py:106-126, 256-266). */
void or_cells(int64_t n, const double* pos, const double* h, double* lo, double* inv,
              int64_t* ncell, int64_t* cell) {
  double box[3] = {0.0, 0.0, 0.0};
  or_grid_geometry(n, pos, h, box, lo, inv, ncell);
  for (int64_t i = 0; i < n; ++i) {
    int64_t cx = cell_of(pos[3 * i + 0], lo[0], inv[0], ncell[0]);
    int64_t cy = cell_of(pos[3 * i + 1], lo[1], inv[1], ncell[1]);
    int64_t cz = cell_of(pos[3 * i + 2], lo[2], inv[2], ncell[2]);
    cell[i] = (cx * ncell[1] + cy) * ncell[2] + cz;
  }
}

void or_free(void* p) { free(p); }

static inline double min_image(double d, double b) {
  if (b > 0.0) d -= b * rint(d / b);
  return d;
}

/* sim/neighbours.py:284-323 (_tighten / tighten): keep r < 2 max(h_i, h_j); rows only.
 * counts (n) is written in the count pass (out_off NULL); the fill pass writes out_idx. */
void or_tighten(int64_t n, const double* pos, const double* h, const double* box,
                const int64_t* offset, const int64_t* index, int64_t nrows, const int64_t* rows,
                int64_t* counts, const int64_t* out_off, int64_t* out_idx) {
  int fill_pass = out_off != NULL;
  if (!fill_pass) memset(counts, 0, sizeof(int64_t) * (size_t)n);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t i = rows[q];
    int64_t m = 0;
    for (int64_t k = offset[i]; k < offset[i + 1]; ++k) {
      int64_t j = index[k];
      double d2 = 0.0;
      for (int c = 0; c < 3; ++c) {
        double dx = min_image(pos[3 * j + c] - pos[3 * i + c], box[c]);
        d2 += dx * dx;
      }
      double rr = R_KERN * (h[i] > h[j] ? h[i] : h[j]);
      if (d2 < rr * rr) {
        if (fill_pass) out_idx[out_off[i] + m] = j;
        m += 1;
      }
    }
    if (!fill_pass) counts[i] = m;
  }
}

/* ------------------------------------------------------------------ density
 * sim/sph.py:215-297 (_sums, _distances, _density_kernel). */
static inline void sums(const double* r, const double* m, int64_t cnt, double h, int kid,
                        double cnorm, double* rs_out, double* dws_out) {
  double rs = 0.0, dws = 0.0;
  double inv_h = 1.0 / h;
  double ih2 = inv_h * inv_h;
  double ih3 = ih2 * inv_h;  /* x**3 and x**4 as Numba evaluates integer powers */
  double ih4 = ih2 * ih2;
  for (int64_t k = 0; k < cnt; ++k) {
    double q = r[k] * inv_h;
    if (q < 2.0) {
      double fq = kernel_f(q, kid);
      rs += m[k] * cnorm * ih3 * fq;
      dws += m[k] * (-cnorm * ih4 * (3.0 * fq + q * kernel_df(q, kid)));
    }
  }
  *rs_out = rs;
  *dws_out = dws;
}

void or_density(int64_t n, const double* pos, const double* mass, const double* h_start,
                const double* h_search, const int64_t* offset, const int64_t* index,
                const double* box, int kid, double cnorm, double eta, double tol, double h_max,
                int64_t nrows, const int64_t* rows, double* h_out, double* rho, double* omega,
                int64_t* iters, int64_t* flags) {
  (void)n;
#pragma omp parallel
  {
    int64_t cap = 0;
    double* r = NULL;
    double* m = NULL;
#pragma omp for schedule(dynamic, 32)
    for (int64_t q = 0; q < nrows; ++q) {
      int64_t i = rows[q];
      double m_i = mass[i];
      int64_t row = offset[i + 1] - offset[i];
      if (row > cap) {
        cap = row * 2 + 16;
        free(r);
        free(m);
        r = (double*)malloc(sizeof(double) * (size_t)cap);
        m = (double*)malloc(sizeof(double) * (size_t)cap);
      }
      double hs = h_search[i] < h_max ? h_search[i] : h_max;
      double r_max = 2.0 * hs;
      int64_t cnt = 0;
      for (int64_t k = offset[i]; k < offset[i + 1]; ++k) {
        int64_t j = index[k];
        double d2 = 0.0;
        for (int c = 0; c < 3; ++c) {
          double dx = min_image(pos[3 * j + c] - pos[3 * i + c], box[c]);
          d2 += dx * dx;
        }
        if (d2 < r_max * r_max) {
          r[cnt] = sqrt(d2);
          m[cnt] = mass[j];
          cnt++;
        }
      }
      double hi = hs, lo = 0.0;
      double h = h_start[i] < hi ? h_start[i] : hi;
      double h0 = h;
      int64_t flag = 3, it = 0;
      double e3 = eta * eta * eta;
      while (it < 50) {
        it += 1;
        double rs, dws;
        sums(r, m, cnt, h, kid, cnorm, &rs, &dws);
        double t = eta / h;
        double f = rs - m_i * (t * t * t);
        double h2 = h * h;
        double df = dws + 3.0 * m_i * e3 / (h2 * h2);
        if (f > 0)
          hi = h;
        else
          lo = h;
        double h_new = df > 0 ? h - f / df : 0.5 * (lo + hi);
        if (!(lo <= h_new && h_new <= hi)) h_new = 0.5 * (lo + hi);
        if (fabs(h_new - h) < tol * h0) {
          h = h_new;
          flag = 0;
          break;
        }
        h = h_new;
      }
      double h_lim = hs;
      if (h >= h_lim * (1 - 1e-3)) {
        double rs_lim, dummy;
        sums(r, m, cnt, h_lim, kid, cnorm, &rs_lim, &dummy);
        double t = eta / h_lim;
        if (rs_lim - m_i * (t * t * t) < 0) {
          h = h_lim;
          flag = h_lim >= h_max ? 1 : 2;
        }
      }
      double rs, dws;
      sums(r, m, cnt, h, kid, cnorm, &rs, &dws);
      h_out[q] = h;
      rho[q] = rs;
      omega[q] = flag == 1 ? 1.0 : 1.0 + h / (3.0 * rs) * dws;
      iters[q] = it;
      flags[q] = flag;
    }
    free(r);
    free(m);
  }
}

/* ------------------------------------------------------------------ forces
 * sim/sph.py:519-652 (_dwdr, _forces_kernel): pressure force, P dV work, signal-velocity
 * viscosity with shock heating (optionally on the reconstructed velocity jump), optional
 * conductivity. */
static inline double dwdr(double r, double h, int kid, double cnorm) {
  double h2 = h * h;
  return cnorm / (h2 * h2) * kernel_df(r / h, kid);
}

/* ------------------------------------------------------------------ gradients
 * sim/sph.py:693-902: corrected gradients dv^k/dx^j = (G R^-1)_kj with
 * R_lj = sum_b m_b (x_b - x_a)^l dW_ab(h_a)/dx_a^j, G_kj = sum_b m_b (v_b - v_a)^k dW/dx_a^j;
 * fewer than 4 list entries, tr R <= 0 or |det R| < 1e-6 (tr R / 3)^3: G / (tr R / 3) instead
 * (0 without neighbours). R^-1 as the adjugate over the determinant. */
#define SINGULAR_TOL 1e-6

static double det3(const double m[9]) {
  return m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
         m[2] * (m[3] * m[7] - m[4] * m[6]);
}

/* out = g R^-1 (or the fallback) for each of ng gradient sums g (3x3, row-major) */
static void corrected(const double rm[9], int64_t cnt, int ng, double* const* g, double* const* out) {
  double scale = (rm[0] + rm[4] + rm[8]) / 3.0;
  double det = det3(rm);
  int singular = cnt < 4 || !(scale > 0.0) || !(fabs(det) >= SINGULAR_TOL * scale * scale * scale);
  if (singular) {
    double inv_s = scale > 0.0 ? 1.0 / scale : 0.0;
    for (int k = 0; k < ng; ++k)
      for (int e = 0; e < 9; ++e) out[k][e] = g[k][e] * inv_s;
    return;
  }
  double ri[9];
  ri[0] = (rm[4] * rm[8] - rm[5] * rm[7]) / det;
  ri[1] = (rm[2] * rm[7] - rm[1] * rm[8]) / det;
  ri[2] = (rm[1] * rm[5] - rm[2] * rm[4]) / det;
  ri[3] = (rm[5] * rm[6] - rm[3] * rm[8]) / det;
  ri[4] = (rm[0] * rm[8] - rm[2] * rm[6]) / det;
  ri[5] = (rm[2] * rm[3] - rm[0] * rm[5]) / det;
  ri[6] = (rm[3] * rm[7] - rm[4] * rm[6]) / det;
  ri[7] = (rm[1] * rm[6] - rm[0] * rm[7]) / det;
  ri[8] = (rm[0] * rm[4] - rm[1] * rm[3]) / det;
  for (int k = 0; k < ng; ++k)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        out[k][3 * i + j] = g[k][3 * i + 0] * ri[0 + j] + g[k][3 * i + 1] * ri[3 + j] +
                            g[k][3 * i + 2] * ri[6 + j];
}

/* sums of one row: R, G (velocities) and, if acc is given, the acceleration gradient sum */
static int64_t gradient_sums(int64_t a, const double* pos, const double* vel, const double* acc,
                             const double* mass, const double* h, const int64_t* offset,
                             const int64_t* index, const double* box, int kid, double cnorm,
                             double rm[9], double gv[9], double ga[9]) {
  for (int e = 0; e < 9; ++e) rm[e] = gv[e] = ga[e] = 0.0;
  int64_t cnt = 0;
  for (int64_t k = offset[a]; k < offset[a + 1]; ++k) {
    int64_t b = index[k];
    if (b == a) continue;
    cnt += 1;
    double dx[3];
    for (int c = 0; c < 3; ++c) dx[c] = min_image(pos[3 * a + c] - pos[3 * b + c], box[c]);
    double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    double g = dwdr(r, h[a], kid, cnorm) / r;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        double gj = mass[b] * g * dx[j];
        rm[3 * i + j] -= dx[i] * gj;
        gv[3 * i + j] += (vel[3 * b + i] - vel[3 * a + i]) * gj;
        if (acc) ga[3 * i + j] += (acc[3 * b + i] - acc[3 * a + i]) * gj;
      }
  }
  return cnt;
}

/* sim/sph.py:850-902 (_gradients_kernel): div v, |curl v| and d(div v)/dt in rows order */
void or_gradients(const double* pos, const double* vel, const double* acc, const double* mass,
                  const double* h, const int64_t* offset, const int64_t* index, const double* box,
                  int kid, double cnorm, int64_t nrows, const int64_t* rows, double* div,
                  double* curl, double* ddiv) {
#pragma omp parallel for schedule(dynamic, 32)
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t a = rows[q];
    double rm[9], gv[9], ga[9], dv[9], da[9];
    int64_t cnt = gradient_sums(a, pos, vel, acc, mass, h, offset, index, box, kid, cnorm, rm, gv, ga);
    double* g[2] = {gv, ga};
    double* o[2] = {dv, da};
    corrected(rm, cnt, 2, g, o);
    div[q] = dv[0] + dv[4] + dv[8];
    double c0 = dv[7] - dv[5], c1 = dv[2] - dv[6], c2 = dv[3] - dv[1];
    curl[q] = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
    double sdd = 0.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) sdd += dv[3 * i + j] * dv[3 * j + i];
    ddiv[q] = da[0] + da[4] + da[8] - sdd;
  }
}

/* sim/sph.py:797-846 (_velocity_gradient_kernel): out[a] = dv/dx (3x3) for a in rows */
void or_velocity_gradients(const double* pos, const double* vel, const double* mass,
                           const double* h, const int64_t* offset, const int64_t* index,
                           const double* box, int kid, double cnorm, int64_t nrows,
                           const int64_t* rows, double* out) {
#pragma omp parallel for schedule(dynamic, 32)
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t a = rows[q];
    double rm[9], gv[9], ga[9];
    int64_t cnt = gradient_sums(a, pos, vel, NULL, mass, h, offset, index, box, kid, cnorm, rm, gv, ga);
    double* g[1] = {gv};
    double* o[1] = {out + 9 * a};
    corrected(rm, cnt, 1, g, o);
  }
}

void or_forces(const double* pos, const double* vel, const double* mass, const double* h,
               const double* rho, const double* omega, const double* pressure, const double* u,
               const double* c_s, const double* alpha, const int64_t* offset,
               const int64_t* index, const double* box, int kid, double cnorm, int use_visc,
               int use_cond, double beta, double alpha_u, int cond_signal, int use_recon,
               int closeness, double eta_crit, double eta_fold, int gate, const double* gvel,
               int64_t nrows, const int64_t* rows, double* acc, double* dudt, double* vsig_max,
               double* vheat, double* cheat) {
#pragma omp parallel for schedule(dynamic, 32)
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t a = rows[q];
    double inv_or_a = 1.0 / (omega[a] * rho[a]);
    double ax = 0.0, ay = 0.0, az = 0.0, work = 0.0, heat = 0.0, visc_heat = 0.0,
           cond_heat = 0.0;
    double vmax = use_visc ? c_s[a] : 0.0;
    for (int64_t k = offset[a]; k < offset[a + 1]; ++k) {
      int64_t b = index[k];
      if (b == a) continue;
      double dx0 = min_image(pos[3 * a + 0] - pos[3 * b + 0], box[0]);
      double dx1 = min_image(pos[3 * a + 1] - pos[3 * b + 1], box[1]);
      double dx2 = min_image(pos[3 * a + 2] - pos[3 * b + 2], box[2]);
      double r = sqrt(dx0 * dx0 + dx1 * dx1 + dx2 * dx2);
      double rx = dx0 / r, ry = dx1 / r, rz = dx2 / r;
      double fa = dwdr(r, h[a], kid, cnorm);
      double fb = dwdr(r, h[b], kid, cnorm);
      double vdotr = (vel[3 * a + 0] - vel[3 * b + 0]) * rx + (vel[3 * a + 1] - vel[3 * b + 1]) * ry +
                     (vel[3 * a + 2] - vel[3 * b + 2]) * rz;
      double num_a = pressure[a], num_b = pressure[b];
      if (use_visc && use_recon) {
        /* physics/viscosity.py:116-158: limiter ratio, van Leer limiter, closeness factor and
         * the jump reconstructed to the pair midpoint (projections G x, x = x_a - x_b) */
        const double* G = gvel + 9 * a;
        const double* H = gvel + 9 * b;
        double ga0 = G[0] * dx0 + G[1] * dx1 + G[2] * dx2;
        double ga1 = G[3] * dx0 + G[4] * dx1 + G[5] * dx2;
        double ga2 = G[6] * dx0 + G[7] * dx1 + G[8] * dx2;
        double gb0 = H[0] * dx0 + H[1] * dx1 + H[2] * dx2;
        double gb1 = H[3] * dx0 + H[4] * dx1 + H[5] * dx2;
        double gb2 = H[6] * dx0 + H[7] * dx1 + H[8] * dx2;
        double pa = dx0 * ga0 + dx1 * ga1 + dx2 * ga2;
        double pb = dx0 * gb0 + dx1 * gb1 + dx2 * gb2;
        double phi = 0.0;
        if (pb != 0.0) {
          double ratio = pa / pb;
          if (ratio > 0.0) phi = fmin(1.0, 4.0 * ratio / ((1.0 + ratio) * (1.0 + ratio)));
        }
        if (closeness) {
          double eta_ab = fmin(r / h[a], r / h[b]);
          if (eta_ab < eta_crit) {
            double t = (eta_ab - eta_crit) / eta_fold;
            phi *= exp(-t * t);
          }
        }
        double vdr = ((vel[3 * a + 0] - 0.5 * phi * ga0) - (vel[3 * b + 0] + 0.5 * phi * gb0)) * rx +
                     ((vel[3 * a + 1] - 0.5 * phi * ga1) - (vel[3 * b + 1] + 0.5 * phi * gb1)) * ry +
                     ((vel[3 * a + 2] - 0.5 * phi * ga2) - (vel[3 * b + 2] + 0.5 * phi * gb2)) * rz;
        int on = vdr < 0.0 && vdotr < 0.0;
        if (gate == 1)
          on = vdr < 0.0;
        else if (gate == 2 && vdotr > vdr)
          vdr = vdotr;
        double vsig_a = alpha[a] * c_s[a] + beta * fabs(vdr);
        double vsig_b = alpha[b] * c_s[b] + beta * fabs(vdr);
        double vsig_cfl = alpha[a] * c_s[a] + beta * fabs(vdotr);
        if (vsig_cfl > vmax) vmax = vsig_cfl;
        if (on) {
          num_a += -0.5 * rho[a] * vsig_a * vdr;
          num_b += -0.5 * rho[b] * vsig_b * vdr;
          double dh = mass[b] * vsig_a * 0.5 * vdr * vdotr * fa * inv_or_a;
          heat -= dh;
          visc_heat -= dh;
        }
      } else if (use_visc) {
        double vsig_a = alpha[a] * c_s[a] + beta * fabs(vdotr);
        double vsig_b = alpha[b] * c_s[b] + beta * fabs(vdotr);
        if (vsig_a > vmax) vmax = vsig_a;
        if (vdotr < 0.0) {
          num_a += -0.5 * rho[a] * vsig_a * vdotr;
          num_b += -0.5 * rho[b] * vsig_b * vdotr;
          double dh = mass[b] * vsig_a * 0.5 * vdotr * vdotr * fa * inv_or_a;
          heat -= dh;
          visc_heat -= dh;
        }
      }
      if (use_cond) {
        double vu;
        if (cond_signal == 0)
          vu = sqrt(fabs(pressure[a] - pressure[b]) / (0.5 * (rho[a] + rho[b])));
        else
          vu = fabs(vdotr);
        double dc = mass[b] * alpha_u * vu * (u[a] - u[b]) * 0.5 *
                    (fa * inv_or_a + fb / (omega[b] * rho[b]));
        heat += dc;
        cond_heat += dc;
      }
      double f = mass[b] * (num_a / (omega[a] * rho[a] * rho[a]) * fa +
                            num_b / (omega[b] * rho[b] * rho[b]) * fb);
      ax -= f * rx;
      ay -= f * ry;
      az -= f * rz;
      work += mass[b] * vdotr * fa;
    }
    acc[3 * q + 0] = ax;
    acc[3 * q + 1] = ay;
    acc[3 * q + 2] = az;
    dudt[q] = pressure[a] * inv_or_a / rho[a] * work + heat;
    vsig_max[q] = vmax;
    vheat[q] = visc_heat;
    cheat[q] = cond_heat;
  }
}

/* sim/sph.py:1084-1117 (_disc_kernel): Lodato-Price disc viscosity on every pair. */
void or_disc_forces(const double* pos, const double* vel, const double* mass, const double* h,
                    const double* rho, const double* omega, const double* c_s, double alpha_av,
                    const int64_t* offset, const int64_t* index, const double* box, int kid,
                    double cnorm, int64_t nrows, const int64_t* rows, double* acc,
                    double* dudt) {
#pragma omp parallel for schedule(dynamic, 32)
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t a = rows[q];
    double ia = 1.0 / (omega[a] * rho[a] * rho[a]);
    double axv[3] = {0.0, 0.0, 0.0}, dx[3];
    double heat = 0.0;
    for (int64_t k = offset[a]; k < offset[a + 1]; ++k) {
      int64_t b = index[k];
      if (b == a) continue;
      for (int c = 0; c < 3; ++c) dx[c] = min_image(pos[3 * a + c] - pos[3 * b + c], box[c]);
      double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      double vdr = 0.0;
      for (int c = 0; c < 3; ++c) vdr += (vel[3 * a + c] - vel[3 * b + c]) * dx[c] / r;
      double qa = -rho[a] * h[a] / (2.0 * r) * alpha_av * c_s[a] * vdr * ia;
      double qb = -rho[b] * h[b] / (2.0 * r) * alpha_av * c_s[b] * vdr / (omega[b] * rho[b] * rho[b]);
      double fa = dwdr(r, h[a], kid, cnorm);
      double fb = dwdr(r, h[b], kid, cnorm);
      double f = mass[b] * (qa * fa + qb * fb);
      for (int c = 0; c < 3; ++c) axv[c] -= f * dx[c] / r;
      heat += mass[b] * qa * vdr * fa;
    }
    for (int c = 0; c < 3; ++c) acc[3 * q + c] = axv[c];
    dudt[q] = heat;
  }
}

/* ------------------------------------------------------------------ GN gravity
 * sim/integrator.py:106-185 (_dh_dx, _dh_dp, _converged, _glf_one, _glf_many_kernel);
 * sim/fastphys.py:24-32 (gn_v_from_p). */
#define GLF_TOL 1e-15
#define GLF_MAX_ITER 10
#define GLF_R_MIN 2.5

static inline void dh_dx(double x0, double x1, double x2, double p0, double p1, double p2,
                         double* g) {
  double r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
  double r2 = r * r, r3 = r2 * r, r4 = r2 * r2, r5 = r4 * r;
  double c = -2.0 * (r - 2.0) / r4;
  double da = 2.0 / (r * r);
  double dc = (6.0 * r - 16.0) / r5;
  double px = p0 * x0 + p1 * x1 + p2 * x2;
  double pp = p0 * p0 + p1 * p1 + p2 * p2;
  double radial = (0.5 * da * pp + 0.5 * dc * px * px) / r + 1.0 / r3;
  g[0] = radial * x0 + c * px * p0;
  g[1] = radial * x1 + c * px * p1;
  g[2] = radial * x2 + c * px * p2;
}

static inline void dh_dp(double x0, double x1, double x2, double p0, double p1, double p2,
                         double* v) {
  double r = sqrt(x0 * x0 + x1 * x1 + x2 * x2);
  double r2 = r * r, r4 = r2 * r2;
  double a = (r - 2.0) / r;
  double c = -2.0 * (r - 2.0) / r4;
  double cpx = c * (p0 * x0 + p1 * x1 + p2 * x2);
  v[0] = a * p0 + cpx * x0;
  v[1] = a * p1 + cpx * x1;
  v[2] = a * p2 + cpx * x2;
}

static inline int converged(const double* nw, const double* old) {
  double d = (nw[0] - old[0]) * (nw[0] - old[0]) + (nw[1] - old[1]) * (nw[1] - old[1]) +
             (nw[2] - old[2]) * (nw[2] - old[2]);
  return d <= GLF_TOL * GLF_TOL * (nw[0] * nw[0] + nw[1] * nw[1] + nw[2] * nw[2]);
}

static int64_t glf_one(const double* x, const double* p, double dt, double* xo, double* po) {
  for (int c = 0; c < 3; ++c) {
    xo[c] = x[c];
    po[c] = p[c];
  }
  if (x[0] * x[0] + x[1] * x[1] + x[2] * x[2] <= GLF_R_MIN * GLF_R_MIN) return -3;
  double half = 0.5 * dt;
  int64_t iters = 0;
  double hp[3] = {p[0], p[1], p[2]}, g[3], nw[3];
  int ok = 0;
  for (int it = 0; it < GLF_MAX_ITER; ++it) {
    dh_dx(x[0], x[1], x[2], hp[0], hp[1], hp[2], g);
    for (int c = 0; c < 3; ++c) nw[c] = p[c] - half * g[c];
    iters += 1;
    ok = converged(nw, hp);
    for (int c = 0; c < 3; ++c) hp[c] = nw[c];
    if (ok) break;
  }
  if (!ok) return -1;
  double v[3], w[3], y[3];
  dh_dp(x[0], x[1], x[2], hp[0], hp[1], hp[2], v);
  for (int c = 0; c < 3; ++c) y[c] = x[c] + dt * v[c];
  ok = 0;
  for (int it = 0; it < GLF_MAX_ITER; ++it) {
    dh_dp(y[0], y[1], y[2], hp[0], hp[1], hp[2], w);
    for (int c = 0; c < 3; ++c) nw[c] = x[c] + half * (v[c] + w[c]);
    iters += 1;
    ok = converged(nw, y);
    for (int c = 0; c < 3; ++c) y[c] = nw[c];
    if (ok) break;
  }
  if (!ok) return -2;
  dh_dx(y[0], y[1], y[2], hp[0], hp[1], hp[2], g);
  for (int c = 0; c < 3; ++c) {
    xo[c] = y[c];
    po[c] = hp[c] - half * g[c];
  }
  return iters;
}

void or_glf_many(int64_t n, const double* x, const double* p, const double* dt, double* x_out,
                 double* p_out, int64_t* iters) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) iters[i] = glf_one(x + 3 * i, p + 3 * i, dt[i], x_out + 3 * i, p_out + 3 * i);
}

void or_gn_v_from_p(int64_t n, const double* x, const double* p, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double v[3];
    dh_dp(x[3 * i], x[3 * i + 1], x[3 * i + 2], p[3 * i], p[3 * i + 1], p[3 * i + 2], v);
    out[3 * i] = v[0];
    out[3 * i + 1] = v[1];
    out[3 * i + 2] = v[2];
  }
}

/* sim/sph.py:85-111 (_fast_rows_complete): brute-force check that every particle within
 * 2 max(h_lim_j, h_lim_k) of a fast particle j is in j's (sorted) list. */
int or_fast_rows_complete(int64_t n, const double* pos, int64_t nfast, const int64_t* fast,
                          const double* h_lim, const double* box, const int64_t* offset,
                          const int64_t* index) {
  for (int64_t q = 0; q < nfast; ++q) {
    int64_t j = fast[q];
    int64_t lo = offset[j], hi = offset[j + 1];
    for (int64_t k = 0; k < n; ++k) {
      double d2 = 0.0;
      for (int c = 0; c < 3; ++c) {
        double dx = min_image(pos[3 * k + c] - pos[3 * j + c], box[c]);
        d2 += dx * dx;
      }
      double rr = 2.0 * (h_lim[j] > h_lim[k] ? h_lim[j] : h_lim[k]);
      if (d2 <= rr * rr) {
        int64_t a = lo, b = hi;
        while (a < b) {
          int64_t m = (a + b) / 2;
          if (index[m] < k)
            a = m + 1;
          else
            b = m;
        }
        if (a >= hi || index[a] != k) return 0;
      }
    }
  }
  return 1;
}

/* sim/blocks.py:337-353 (_limit_rows): raise the levels of rows until each is within max_gap
 * of every neighbour's (Gauss-Seidel sweeps until nothing changes). */
void or_limit_rows(int64_t* level, int64_t nrows, const int64_t* rows, const int64_t* offset,
                   const int64_t* index, int64_t max_gap) {
  int changed = 1;
  while (changed) {
    changed = 0;
    for (int64_t q = 0; q < nrows; ++q) {
      int64_t i = rows[q];
      int64_t need = level[i];
      for (int64_t k = offset[i]; k < offset[i + 1]; ++k) {
        int64_t j = index[k];
        if (level[j] - max_gap > need) need = level[j] - max_gap;
      }
      if (need > level[i]) {
        level[i] = need;
        changed = 1;
      }
    }
  }
}

/* sim/blocks.py:356-364 (_wake_targets). */
void or_wake_targets(const int64_t* level, int64_t nrows, const int64_t* rows,
                     const int64_t* offset, const int64_t* index, int64_t max_gap,
                     int64_t* need) {
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t i = rows[q];
    for (int64_t k = offset[i]; k < offset[i + 1]; ++k) {
      int64_t j = index[k];
      if (level[i] - max_gap > need[j]) need[j] = level[i] - max_gap;
    }
  }
}

/* sim/blocks.py:201-214 (_mark_neighbours). */
void or_mark_neighbours(int64_t nrows, const int64_t* rows, const int64_t* offset,
                        const int64_t* index, uint8_t* mark) {
  for (int64_t q = 0; q < nrows; ++q) {
    int64_t i = rows[q];
    mark[i] = 1;
    for (int64_t k = offset[i]; k < offset[i + 1]; ++k) mark[index[k]] = 1;
  }
}

/* sim/fastphys.py:45-71 (_gasrad_t_kernel): T [K] of gas + radiation from rho [kg/m^3] and
 * u [J/kg] by Newton on log T inside the bracket [1, 1e13] K narrowed every iteration, tolerance
 * 1e-12, at most 200 iterations; ok[i] = 0 where it does not converge.  t**4 is evaluated by
 * squaring, as Numba lowers it. */
void or_gasrad_temperature(int64_t n, const double* rho, const double* u, double a1, double a_rad,
                           double* out, uint8_t* ok) {
  const double lt_min = log(1.0), lt_max = log(1.0e13);
  const double t_min = exp(lt_min), t_max = exp(lt_max);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    const double r = rho[i], uu = u[i];
    double lo = lt_min, hi = lt_max;
    double t0 = fmin(uu / a1, pow(uu * r / a_rad, 0.25));
    double lt = log(fmin(fmax(t0, t_min), t_max));
    ok[i] = 0;
    for (int it = 0; it < 200; ++it) {
      double t = exp(lt);
      double t2 = t * t;
      double t4 = t2 * t2;
      double f = a1 * t + a_rad * t4 / r - uu;
      double dfdl = a1 * t + 4.0 * a_rad * t4 / r;
      if (f < 0) lo = lt;
      if (f > 0) hi = lt;
      double nw = lt - f / dfdl;
      if (nw <= lo || nw >= hi || !isfinite(nw)) nw = 0.5 * (lo + hi);
      double step = fabs(nw - lt);
      lt = nw;
      if (step < 1e-12) {
        ok[i] = 1;
        break;
      }
    }
    out[i] = exp(lt);
  }
}

/* ------------------------------------------------------------------ grid deposition
 * render/gasgrid.py:316-532 (_nb_log_kernel_pass, _nb_log_deposit_chunk) and 534-597
 * (_nb_box_deposit_chunk): each particle's fields vals (6 per particle: m, m T, m T^4, m v)
 * go to the cells whose centres lie inside its support (q < 2), weighted by f(q) V_c and
 * normalised; fewer than 8 such centres: trilinear weights in index space.  Particles are dealt
 * to nchunk chunks in turn (p -> chunk p mod nchunk) into separate grids, summed in order, as
 * the reference does (render/gasgrid.py:660-676). */
#define DEP_FIELDS 6
#define DEP_MIN_CELLS 8
#define DEP_INNER_VIRTUAL 64

static double dep_kernel_f(double q, int kid) {
  if (q >= 2.0) return 0.0;
  if (kid == 0) {
    if (q < 1.0) return 1.0 - 1.5 * q * q + 0.75 * q * q * q;
    double t = 2.0 - q;
    return 0.25 * t * t * t;
  }
  double x = 1.0 - 0.5 * q;
  double x2 = x * x;
  return x2 * x2 * x2 * (35.0 / 12.0 * q * q + 3.0 * q + 1.0);
}

typedef struct {
  double r_min, dlnr, dth, dph;
  int nr, nth, nph;
  const double *sth, *cth, *dcth, *cph, *sph;
} dep_log_grid;

/* one pass over the centres inside the support; mode 0 counts and sums f V, mode 1 adds */
static void dep_log_pass(const dep_log_grid* g, double xp, double yp, double zp, double rr,
                         double th, double ph, double hp, int i_lo, int i_hi, int kid, int mode,
                         double inv, const double* vals, double m, double* acc, double* wsum,
                         int64_t* n_in, double* outside) {
  double big = 2.0 * hp;
  double ct0 = cos(th), st0 = sin(th);
  for (int i = i_lo; i <= i_hi; ++i) {
    double rc = g->r_min * exp((i + 0.5) * g->dlnr);
    double cos_a = (rc * rc + rr * rr - big * big) / (2.0 * rc * rr);
    if (cos_a > 1.0) continue;
    int j0, j1;
    if (cos_a <= -1.0) {
      j0 = 0;
      j1 = g->nth - 1;
    } else {
      double a = acos(cos_a);
      j0 = (int)floor((th - a) / g->dth) - 1;
      if (j0 < 0) j0 = 0;
      j1 = (int)floor((th + a) / g->dth) + 1;
      if (j1 > g->nth - 1) j1 = g->nth - 1;
    }
    double r1 = g->r_min * exp(i * g->dlnr);
    double r2 = r1 * exp(g->dlnr);
    double vr = (r2 * r2 * r2 - r1 * r1 * r1) / 3.0;
    int ing = 0 <= i && i < g->nr;
    for (int j = j0; j <= j1; ++j) {
      double ss = st0 * g->sth[j];
      int full = 1;
      int k0 = 0, k1 = g->nph - 1;
      if (ss > 1e-300 && cos_a > -1.0) {
        double cd = (cos_a - ct0 * g->cth[j]) / ss;
        if (cd > 1.0 + 1e-12) continue;
        if (cd > -1.0) {
          double dp = acos(fmin(cd, 1.0));
          k0 = (int)ceil((ph - dp) / g->dph - 0.5) - 1;
          k1 = (int)floor((ph + dp) / g->dph - 0.5) + 1;
          if (k1 - k0 + 1 < g->nph) full = 0;
        }
      }
      if (full) {
        k0 = 0;
        k1 = g->nph - 1;
      }
      double rst = rc * g->sth[j];
      double dzc = rc * g->cth[j] - zp;
      double vrt = vr * g->dcth[j] * g->dph;
      for (int kk = k0; kk <= k1; ++kk) {
        int k = ((kk % g->nph) + g->nph) % g->nph;
        double dxc = rst * g->cph[k] - xp;
        double dyc = rst * g->sph[k] - yp;
        double q = sqrt(dxc * dxc + dyc * dyc + dzc * dzc) / hp;
        if (q < 2.0) {
          if (mode == 0) {
            *n_in += 1;
            *wsum += dep_kernel_f(q, kid) * vrt;
          } else {
            double w = dep_kernel_f(q, kid) * vrt * inv;
            if (ing) {
              double* c = acc + (((int64_t)i * g->nth + j) * g->nph + k) * DEP_FIELDS;
              for (int f = 0; f < DEP_FIELDS; ++f) c[f] += w * vals[f];
            } else {
              *outside += w * m;
            }
          }
        }
      }
    }
  }
}

static double py_mod(double a, double b) {  /* Python's a % b for b > 0 */
  double r = fmod(a, b);
  if (r != 0.0 && r < 0.0) r += b;
  return r;
}

static int py_imod(int a, int b) { return ((a % b) + b) % b; }

void or_deposit_log(int64_t n, const double* x, const double* h, const double* m,
                    const double* vals, double r_min, double dlnr, double dth, double dph, int nr,
                    int nth, int nph, int kid, const double* sth, const double* cth,
                    const double* dcth, const double* cph, const double* sph, int nchunk,
                    double* acc, double* outside_out, int64_t* n_tri_out) {
  dep_log_grid g = {r_min, dlnr, dth, dph, nr, nth, nph, sth, cth, dcth, cph, sph};
  const int64_t ncell = (int64_t)nr * nth * nph * DEP_FIELDS;
  double* part = (double*)calloc((size_t)ncell * nchunk, sizeof(double));
  double outside = 0.0;
  int64_t n_tri = 0;
  double lnr0 = log(r_min);
  double two_pi = 2.0 * 3.141592653589793;
  for (int c = 0; c < nchunk; ++c) {
    double* a = part + ncell * c;
    double out_c = 0.0;
    for (int64_t p = c; p < n; p += nchunk) {
      double xp = x[3 * p], yp = x[3 * p + 1], zp = x[3 * p + 2];
      double rr = sqrt(xp * xp + yp * yp + zp * zp);
      double hp = h[p];
      double big = 2.0 * hp;
      int i_hi = (int)floor((log(rr + big) - lnr0) / dlnr);
      int i_lo;
      if (big >= rr) {
        i_lo = -DEP_INNER_VIRTUAL;
      } else {
        i_lo = (int)floor((log(rr - big) - lnr0) / dlnr);
        if (i_lo < -DEP_INNER_VIRTUAL) i_lo = -DEP_INNER_VIRTUAL;
      }
      double th = acos(fmin(1.0, fmax(-1.0, zp / rr)));
      double ph = py_mod(atan2(yp, xp), two_pi);
      double wsum = 0.0, dummy = 0.0;
      int64_t n_in = 0;
      dep_log_pass(&g, xp, yp, zp, rr, th, ph, hp, i_lo, i_hi, kid, 0, 0.0, vals + 6 * p, m[p],
                   a, &wsum, &n_in, &dummy);
      if (n_in >= DEP_MIN_CELLS) {
        double o = 0.0;
        int64_t dn = 0;
        dep_log_pass(&g, xp, yp, zp, rr, th, ph, hp, i_lo, i_hi, kid, 1, 1.0 / wsum,
                     vals + 6 * p, m[p], a, &dummy, &dn, &o);
        out_c += o;
        continue;
      }
      n_tri += 1;
      double fr = log(rr / r_min) / dlnr - 0.5;
      double fth = th / dth - 0.5;
      double fph = ph / dph - 0.5;
      int i0 = (int)floor(fr), j0 = (int)floor(fth), k0 = (int)floor(fph);
      double ti = fr - i0, tj = fth - j0, tk = fph - k0;
      if (j0 < 0) {
        j0 = 0;
        tj = 0.0;
      }
      if (j0 > nth - 2) {
        j0 = nth - 2;
        tj = 1.0;
      }
      for (int di = 0; di < 2; ++di) {
        double wi = di == 1 ? ti : 1.0 - ti;
        for (int dj = 0; dj < 2; ++dj) {
          double wj = dj == 1 ? tj : 1.0 - tj;
          for (int dk = 0; dk < 2; ++dk) {
            double wk = dk == 1 ? tk : 1.0 - tk;
            double w = wi * wj * wk;
            int i = i0 + di;
            if (0 <= i && i < nr) {
              int k = py_imod(k0 + dk, nph);
              double* cc = a + (((int64_t)i * nth + j0 + dj) * nph + k) * DEP_FIELDS;
              for (int f = 0; f < DEP_FIELDS; ++f) cc[f] += w * vals[6 * p + f];
            } else {
              out_c += w * m[p];
            }
          }
        }
      }
    }
    outside += out_c;
  }
  for (int64_t e = 0; e < ncell; ++e) {
    double s = part[e];
    for (int c = 1; c < nchunk; ++c) s += part[ncell * c + e];
    acc[e] = s;
  }
  free(part);
  *outside_out = outside;
  *n_tri_out = n_tri;
}

void or_deposit_box(int64_t n, const double* x, const double* h, const double* m,
                    const double* vals, double x0, double y0, double z0, double dx, int nb,
                    int kid, int nchunk, double* acc, double* outside_out, int64_t* n_tri_out) {
  const int64_t ncell = (int64_t)nb * nb * nb * DEP_FIELDS;
  double* part = (double*)calloc((size_t)ncell * nchunk, sizeof(double));
  double outside = 0.0;
  int64_t n_tri = 0;
  for (int c = 0; c < nchunk; ++c) {
    double* A = part + ncell * c;
    double out_c = 0.0;
    for (int64_t p = c; p < n; p += nchunk) {
      double xp = x[3 * p], yp = x[3 * p + 1], zp = x[3 * p + 2];
      double hp = h[p];
      double big = 2.0 * hp;
      int a0 = (int)floor((xp - big - x0) / dx), a1 = (int)floor((xp + big - x0) / dx);
      int b0 = (int)floor((yp - big - y0) / dx), b1 = (int)floor((yp + big - y0) / dx);
      int c0 = (int)floor((zp - big - z0) / dx), c1 = (int)floor((zp + big - z0) / dx);
      double wsum = 0.0;
      int64_t n_in = 0;
      for (int a = a0; a <= a1; ++a) {
        double dxc = x0 + (a + 0.5) * dx - xp;
        for (int b = b0; b <= b1; ++b) {
          double dyc = y0 + (b + 0.5) * dx - yp;
          for (int cz = c0; cz <= c1; ++cz) {
            double dzc = z0 + (cz + 0.5) * dx - zp;
            double q = sqrt(dxc * dxc + dyc * dyc + dzc * dzc) / hp;
            if (q < 2.0) {
              n_in += 1;
              wsum += dep_kernel_f(q, kid);
            }
          }
        }
      }
      if (n_in >= DEP_MIN_CELLS) {
        double inv = 1.0 / wsum;
        for (int a = a0; a <= a1; ++a) {
          double dxc = x0 + (a + 0.5) * dx - xp;
          for (int b = b0; b <= b1; ++b) {
            double dyc = y0 + (b + 0.5) * dx - yp;
            for (int cz = c0; cz <= c1; ++cz) {
              double dzc = z0 + (cz + 0.5) * dx - zp;
              double q = sqrt(dxc * dxc + dyc * dyc + dzc * dzc) / hp;
              if (q < 2.0) {
                double w = dep_kernel_f(q, kid) * inv;
                if (0 <= a && a < nb && 0 <= b && b < nb && 0 <= cz && cz < nb) {
                  double* cc = A + (((int64_t)a * nb + b) * nb + cz) * DEP_FIELDS;
                  for (int f = 0; f < DEP_FIELDS; ++f) cc[f] += w * vals[6 * p + f];
                } else {
                  out_c += w * m[p];
                }
              }
            }
          }
        }
        continue;
      }
      n_tri += 1;
      double fa = (xp - x0) / dx - 0.5, fb = (yp - y0) / dx - 0.5, fc = (zp - z0) / dx - 0.5;
      int ia = (int)floor(fa), ib = (int)floor(fb), ic = (int)floor(fc);
      double ta = fa - ia, tb = fb - ib, tc = fc - ic;
      for (int da = 0; da < 2; ++da) {
        double wa = da == 1 ? ta : 1.0 - ta;
        for (int db = 0; db < 2; ++db) {
          double wb = db == 1 ? tb : 1.0 - tb;
          for (int dc = 0; dc < 2; ++dc) {
            double wc = dc == 1 ? tc : 1.0 - tc;
            double w = wa * wb * wc;
            int a = ia + da, b = ib + db, cz = ic + dc;
            if (0 <= a && a < nb && 0 <= b && b < nb && 0 <= cz && cz < nb) {
              double* cc = A + (((int64_t)a * nb + b) * nb + cz) * DEP_FIELDS;
              for (int f = 0; f < DEP_FIELDS; ++f) cc[f] += w * vals[6 * p + f];
            } else {
              out_c += w * m[p];
            }
          }
        }
      }
    }
    outside += out_c;
  }
  for (int64_t e = 0; e < ncell; ++e) {
    double s = part[e];
    for (int c = 1; c < nchunk; ++c) s += part[ncell * c + e];
    acc[e] = s;
  }
  free(part);
  *outside_out = outside;
  *n_tri_out = n_tri;
}
