// ============================================================================
//  tf_oracle.cpp -- CPU restatement of T-Flows' native Krylov path.
//
//  TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path is
//  compared against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
//  baseline leg load it; the product library (libtfkrylov.so) never links it
//  and never falls back to it.
//
//  PINNED TO THE REFERENCE: the reference is Fortran 2008 and no Fortran
//  compiler is available, so its source is executed instead by
//  oracle/f90exec.py (a translator of the Fortran subset the path's files
//  use); the golden fixtures are that execution's outputs, and this
//  restatement reproduces them bit for bit, as it does the executed source
//  on every case of tests/test_reference_exec.py.  Further pins: scipy's
//  independent PCG, compared iterate by iterate, the identity
//  Bicg(A) == Cg(A) bitwise (Bicg.f90:129-133 copies r1 into r2 and never
//  uses A^T), the 4x4 CSR example of Matrix_Mod.f90:44-55, and a pure-Python
//  line-by-line transliteration (oracle/pyref.py).
//
//  Conventions follow the reference exactly:
//    * all `real` are FP64 (REAL=double build, makefile -fdefault-real-8);
//    * row/col/dia/pos hold 1-based indices, as Matrix_Type stores them;
//      C pointers point at element 1 (x1[k-1] == x(k));
//    * loop orders are those of the Fortran loops, and every `!$omp parallel
//      do` site of the reference is an `omp parallel for` here.  With one
//      OpenMP thread every sum is the reference's serial sum, bit for bit;
//    * built with -ffp-contract=off because the reference's gnu build uses
//      -O3 without -march (x86-64 baseline, no FMA), so a*b+c rounds twice.
//
//  Files restated (paths inside the T-Flows tree):
//    Sources/Process/Cpu/Native_Mod/Cg.f90, Bicg.f90, Prec_Form.f90,
//    Prec_Solve.f90, Residual_Vector.f90, Normalized_Root_Mean_Square.f90,
//    Root_Mean_Square.f90, Solve_Native.f90;
//    Sources/Process/Cpu/Solver_Mod/Set_Singular.f90;
//    Sources/Process/Cpu/Matrix_Mod/Create_Matrix.f90;
//    Sources/Process/Cpu/Process_Mod/Rhie_And_Chow.f90:195-206 (pressure),
//    Compute_Momentum.f90:270-297 and Numerics_Mod/Inertial_Term.f90
//    (momentum) -- used for assembling synthetic systems.
// ============================================================================
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Sources/Shared/Const_Mod.f90:84-93
const double TF_MICRO = 1.0e-6;
const double TF_TINY  = 1.0e-15;
const double TF_HUGE  = 1.0e+15;

enum { PREC_NONE = 0, PREC_JACOBI = 1, PREC_ICC = 2 };

// Fortran min/max on reals: result is the second argument when the first
// compares false (gfortran evaluates max(a,b) as a > b ? a : b for these).
inline double fmin_f(double a, double b) { return (b < a) ? b : a; }
inline double fmax_f(double a, double b) { return (b > a) ? b : a; }

struct Csr {
  int nt, ni;
  const int* row;    // row(1..nt+1)
  const int* col;    // col(1..nnz)
  const int* dia;    // dia(1..nt)
  double*    val;    // val(1..nnz), modified in place by the solvers
  int R(int i) const { return row[i - 1]; }
  int C(int j) const { return col[j - 1]; }
  int D(int i) const { return dia[i - 1]; }
  double& V(int j) const { return val[j - 1]; }
};

// Normalized_Root_Mean_Square.f90:33-63 (serial sum: no omp in the reference)
double nrms(const Csr& A, int ni, const double* r, const double* x,
            int has_norm, double norm) {
  double rms = 0.0;
  for (int i = 1; i <= ni; ++i) {
    double ri = r[i - 1];
    double ai = A.V(A.D(i));
    rms = rms + (ri * ri) / (ai * ai);
  }
  // Global % Sum_Real: no-op on one process
  rms = std::sqrt(rms);
  double x_min, x_max;
  if (!has_norm) {
    x_min = +TF_HUGE;
    x_max = -TF_HUGE;
    for (int i = 1; i <= ni; ++i) {
      x_min = fmin_f(x_min, x[i - 1]);
      x_max = fmax_f(x_max, x[i - 1]);
    }
  } else {
    x_min = 0.0;
    x_max = norm;
  }
  double x_max_min = x_max - x_min;
  x_max_min = fmax_f(x_max_min, TF_TINY);
  rms = rms / x_max_min;
  return rms;
}

// Root_Mean_Square.f90:22-32
double rms_plain(int ni, const double* r) {
  double rms = 0.0;
#pragma omp parallel for reduction(+ : rms)
  for (int i = 1; i <= ni; ++i) rms = rms + r[i - 1] * r[i - 1];
  return std::sqrt(rms);
}

// Residual_Vector.f90:34-42
void residual_vector(const Csr& A, int ni, double* r, const double* b,
                     const double* x) {
#pragma omp parallel for
  for (int i = 1; i <= ni; ++i) {
    double ri = b[i - 1];
    for (int j = A.R(i); j <= A.R(i + 1) - 1; ++j) {
      int k = A.C(j);
      ri = ri - A.V(j) * x[k - 1];
    }
    r[i - 1] = ri;
  }
}

// Prec_Form.f90:47-89
void prec_form(const Csr& A, int ni, double* d, double* d_inv, int prec) {
  if (prec == PREC_JACOBI) {
#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) {
      d[i - 1] = A.V(A.D(i));
      d_inv[i - 1] = 1.0 / d[i - 1];
    }
  } else if (prec == PREC_ICC) {
    for (int i = 1; i <= ni; ++i) {
      double sum = A.V(A.D(i));
      for (int j = A.R(i) + 1; j <= A.R(i + 1) - 1; ++j) {
        int k = A.C(j);
        if (k > i) break;
        sum = sum - d[k - 1] * A.V(j) * A.V(j);
      }
      d_inv[i - 1] = sum;
      d[i - 1] = 1.0 / sum;
    }
  } else {
#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) d[i - 1] = 1.0;
  }
}

// Prec_Solve.f90:44-102
void prec_solve(const Csr& A, int ni, const double* d, const double* d_inv,
                double* x, const double* b, int prec) {
  if (prec == PREC_JACOBI) {
#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) x[i - 1] = b[i - 1] * d_inv[i - 1];
  } else if (prec == PREC_ICC) {
    for (int i = 1; i <= ni; ++i) {          // forward substitution
      double sum = b[i - 1];
      for (int j = A.R(i) + 1; j <= A.R(i + 1) - 1; ++j) {
        int k = A.C(j);
        if (k > i) break;
        sum = sum - A.V(j) * x[k - 1];
      }
      x[i - 1] = sum * d[i - 1];
    }
#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) x[i - 1] = x[i - 1] * d_inv[i - 1];
    for (int i = ni; i >= 1; --i) {          // backward substitution
      double sum = x[i - 1];
      for (int j = A.R(i + 1) - 1; j >= A.R(i) + 1; --j) {
        int k = A.C(j);
        if (k < i) break;
        if (k <= ni) sum = sum - A.V(j) * x[k - 1];
      }
      x[i - 1] = sum * d[i - 1];
    }
  } else {
#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) x[i - 1] = b[i - 1];
  }
}

// Normalisation of Cg.f90:62-84 / Bicg.f90:63-85; returns fn
double normalize(const Csr& A, double* b) {
  double sum_a = 0.0;
  int sum_n = 0;
#pragma omp parallel for reduction(+ : sum_a) reduction(+ : sum_n)
  for (int i = 1; i <= A.ni; ++i) {
    sum_a = sum_a + A.V(A.D(i));
    sum_n = sum_n + 1;
  }
  sum_a = sum_a / (double)sum_n;
  double fn = 1.0 / sum_a;
#pragma omp parallel for
  for (int i = 1; i <= A.nt; ++i) {
    for (int j = A.R(i); j <= A.R(i + 1) - 1; ++j) A.V(j) = A.V(j) * fn;
    b[i - 1] = b[i - 1] * fn;
  }
  return fn;
}

// De-normalisation of Cg.f90:245-250 / Bicg.f90:255-262
void denormalize(const Csr& A, double* b, double fn) {
#pragma omp parallel for
  for (int i = 1; i <= A.nt; ++i) {
    for (int j = A.R(i); j <= A.R(i + 1) - 1; ++j) A.V(j) = A.V(j) / fn;
    b[i - 1] = b[i - 1] / fn;
  }
}

// Cg.f90:2-257.  hist (optional, miter+1 entries) receives res before the
// loop and after each iteration; hist entries not reached are left alone.
void cg(const Csr& A, double* x, double* b, int prec, int miter, int* niter,
        double tol, double* fin_res, int has_norm, double norm,
        double* hist) {
  const int nt = A.nt, ni = A.ni;
  std::vector<double> p1(nt), q1(nt), r1(nt), d(nt), d_inv(nt);
  double alfa, beta, rho, rho_old = 0.0, bnrm2, res;
  int iter;

  res = 0.0;
  double fn = normalize(A, b);
  prec_form(A, ni, d.data(), d_inv.data(), prec);

  bnrm2 = nrms(A, ni, b, x, has_norm, norm);
  if (bnrm2 < tol) { iter = 0; goto done; }

  residual_vector(A, ni, r1.data(), b, x);
  res = nrms(A, ni, r1.data(), x, has_norm, norm);
  if (hist) hist[0] = res;
  if (res < tol) { iter = 0; goto done; }

#pragma omp parallel for
  for (int i = 1; i <= ni; ++i) p1[i - 1] = r1[i - 1];

  for (iter = 1; iter <= miter; ++iter) {
    prec_solve(A, ni, d.data(), d_inv.data(), q1.data(), r1.data(), prec);

    rho = 0.0;
#pragma omp parallel for reduction(+ : rho)
    for (int i = 1; i <= ni; ++i) rho = rho + q1[i - 1] * r1[i - 1];

    if (iter == 1) {
#pragma omp parallel for
      for (int i = 1; i <= ni; ++i) p1[i - 1] = q1[i - 1];
    } else {
      beta = rho / rho_old;
#pragma omp parallel for
      for (int i = 1; i <= ni; ++i) p1[i - 1] = q1[i - 1] + beta * p1[i - 1];
    }

#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) {
      double qi = 0.0;
      for (int j = A.R(i); j <= A.R(i + 1) - 1; ++j) {
        int k = A.C(j);
        qi = qi + A.V(j) * p1[k - 1];
      }
      q1[i - 1] = qi;
    }

    alfa = 0.0;
#pragma omp parallel for reduction(+ : alfa)
    for (int i = 1; i <= ni; ++i) alfa = alfa + p1[i - 1] * q1[i - 1];
    alfa = rho / alfa;

#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) {
      x[i - 1] = x[i - 1] + alfa * p1[i - 1];
      r1[i - 1] = r1[i - 1] - alfa * q1[i - 1];
    }

    res = nrms(A, ni, r1.data(), x, has_norm, norm);
    if (hist) hist[iter] = res;
    if (res < tol) goto done;
    rho_old = rho;
  }
  iter = iter - 1;   // Fortran leaves the do variable at miter+1

done:
  denormalize(A, b, fn);
  *fin_res = res;
  *niter = iter;
}

// Bicg.f90:2-269
void bicg(const Csr& A, double* x, double* b, int prec, int miter, int* niter,
          double tol, double* fin_res, int has_norm, double norm,
          double* hist) {
  const int nt = A.nt, ni = A.ni;
  std::vector<double> p1(nt), q1(nt), r1(nt), p2(nt), q2(nt), r2(nt), d(nt),
      d_inv(nt);
  double alfa, beta, rho, rho_old = 0.0, bnrm2, res;
  int iter;

  res = 0.0;
  double fn = normalize(A, b);
  prec_form(A, ni, d.data(), d_inv.data(), prec);

  bnrm2 = nrms(A, ni, b, x, has_norm, norm);
  if (bnrm2 < tol) { iter = 0; goto done; }

  residual_vector(A, ni, r1.data(), b, x);
  res = nrms(A, ni, r1.data(), x, has_norm, norm);
  if (hist) hist[0] = res;
  if (res < tol) { iter = 0; goto done; }

#pragma omp parallel for
  for (int i = 1; i <= ni; ++i) r2[i - 1] = r1[i - 1];

  for (iter = 1; iter <= miter; ++iter) {
    prec_solve(A, ni, d.data(), d_inv.data(), q1.data(), r1.data(), prec);
    prec_solve(A, ni, d.data(), d_inv.data(), q2.data(), r2.data(), prec);

    rho = 0.0;
#pragma omp parallel for reduction(+ : rho)
    for (int i = 1; i <= ni; ++i) rho = rho + q1[i - 1] * r2[i - 1];

    if (iter == 1) {
#pragma omp parallel for
      for (int i = 1; i <= ni; ++i) {
        p1[i - 1] = q1[i - 1];
        p2[i - 1] = q2[i - 1];
      }
    } else {
      beta = rho / rho_old;
#pragma omp parallel for
      for (int i = 1; i <= ni; ++i) {
        p1[i - 1] = q1[i - 1] + beta * p1[i - 1];
        p2[i - 1] = q2[i - 1] + beta * p2[i - 1];
      }
    }

#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) {
      double a1 = 0.0, a2 = 0.0;
      for (int j = A.R(i); j <= A.R(i + 1) - 1; ++j) {
        int k = A.C(j);
        a1 = a1 + A.V(j) * p1[k - 1];
        a2 = a2 + A.V(j) * p2[k - 1];
      }
      q1[i - 1] = a1;
      q2[i - 1] = a2;
    }

    alfa = 0.0;
#pragma omp parallel for reduction(+ : alfa)
    for (int i = 1; i <= ni; ++i) alfa = alfa + p2[i - 1] * q1[i - 1];
    alfa = rho / alfa;

#pragma omp parallel for
    for (int i = 1; i <= ni; ++i) {
      x[i - 1] = x[i - 1] + alfa * p1[i - 1];
      r1[i - 1] = r1[i - 1] - alfa * q1[i - 1];
      r2[i - 1] = r2[i - 1] - alfa * q2[i - 1];
    }

    res = nrms(A, ni, r1.data(), x, has_norm, norm);
    if (hist) hist[iter] = res;
    if (res < tol) goto done;
    rho_old = rho;
  }
  iter = iter - 1;

done:
  denormalize(A, b, fn);
  *fin_res = res;
  *niter = iter;
}

}  // namespace

extern "C" {

// Number of OpenMP threads; 1 gives the reference's serial sums bit for bit.
void tfo_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

int tfo_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Solve_Native.f90:33-44.  solver: 0 = 'cg', 1 = 'bicg'; prec: 0 none,
// 1 jacobi, 2 icc.  Returns 0, or 64 for an unknown solver (the reference's
// Message % Error(64, ...) code).  x points at x(1), b at b(1).
int tfo_solve_native(int solver, int prec, int nt, int ni, const int* row,
                     const int* col, const int* dia, double* val, double* x,
                     double* b, int miter, int* niter, double tol,
                     double* fin_res, int has_norm, double norm,
                     double* hist) {
  Csr A{nt, ni, row, col, dia, val};
  if (solver == 1)
    bicg(A, x, b, prec, miter, niter, tol, fin_res, has_norm, norm, hist);
  else if (solver == 0)
    cg(A, x, b, prec, miter, niter, tol, fin_res, has_norm, norm, hist);
  else
    return 64;
  return 0;
}

double tfo_nrms(int nt, int ni, const int* row, const int* col,
                const int* dia, double* val, const double* r,
                const double* x, int has_norm, double norm) {
  Csr A{nt, ni, row, col, dia, val};
  return nrms(A, ni, r, x, has_norm, norm);
}

double tfo_rms(int ni, const double* r) { return rms_plain(ni, r); }

void tfo_residual_vector(int nt, int ni, const int* row, const int* col,
                         const int* dia, double* val, double* r,
                         const double* b, const double* x) {
  Csr A{nt, ni, row, col, dia, val};
  residual_vector(A, ni, r, b, x);
}

// One q = A p exactly as the Cg main loop computes it (Cg.f90:177-185).
void tfo_spmv(int nt, int ni, const int* row, const int* col, const int* dia,
              double* val, const double* p, double* q) {
  Csr A{nt, ni, row, col, dia, val};
#pragma omp parallel for
  for (int i = 1; i <= ni; ++i) {
    double qi = 0.0;
    for (int j = A.R(i); j <= A.R(i + 1) - 1; ++j)
      qi = qi + A.V(j) * p[A.C(j) - 1];
    q[i - 1] = qi;
  }
}

void tfo_prec_form(int nt, int ni, const int* row, const int* col,
                   const int* dia, double* val, double* d, double* d_inv,
                   int prec) {
  Csr A{nt, ni, row, col, dia, val};
  prec_form(A, ni, d, d_inv, prec);
}

void tfo_prec_solve(int nt, int ni, const int* row, const int* col,
                    const int* dia, double* val, const double* d,
                    const double* d_inv, double* x, const double* b,
                    int prec) {
  Csr A{nt, ni, row, col, dia, val};
  prec_solve(A, ni, d, d_inv, x, b, prec);
}

// Set_Singular.f90:29-31 (native branch)
void tfo_set_singular(int n_cells, const int* dia, double* val) {
  for (int i = 1; i <= n_cells; ++i)
    val[dia[i - 1] - 1] = val[dia[i - 1] - 1] * (1.0 + TF_MICRO);
}

// Create_Matrix.f90:45-139.  faces_c is (2, n_faces) column-major: faces_c[2s]
// = c1, faces_c[2s+1] = c2 (1-based, c2 <= 0 on boundaries).  Returns nnz
// (without the +1 pad of :80-82).  row must hold n_cells+1 ints, col and
// nnz_cap ints, dia n_cells, pos 2*n_faces.  Returns -1 if nnz_cap is too
// small, -2 if a diagonal is not first (the Assert at :118).
long tfo_create_matrix(int n_cells, int n_faces, const int* faces_c,
                       int* row, int* col, long nnz_cap, int* dia, int* pos) {
  std::vector<int> stencw(n_cells + 1, 1);
  for (int s = 1; s <= n_faces; ++s) {
    int c1 = faces_c[2 * (s - 1)], c2 = faces_c[2 * (s - 1) + 1];
    if (c2 > 0) { stencw[c1]++; stencw[c2]++; }
  }
  long n = 0;
  for (int c = 1; c <= n_cells; ++c) n += stencw[c];
  if (n > nnz_cap) return -1;
  for (long j = 0; j < n; ++j) col[j] = 0;
  for (int c = 0; c < n_cells; ++c) dia[c] = 0;
  for (long s = 0; s < 2L * n_faces; ++s) pos[s] = 0;

  row[0] = 1;
  for (int c = 1; c <= n_cells; ++c) {
    row[c] = row[c - 1] + stencw[c];
    col[row[c - 1] - 1] = c;
    stencw[c] = 1;
  }
  for (int s = 1; s <= n_faces; ++s) {
    int c1 = faces_c[2 * (s - 1)], c2 = faces_c[2 * (s - 1) + 1];
    if (c2 > 0) {
      col[row[c1 - 1] + stencw[c1] - 1] = c2;
      col[row[c2 - 1] + stencw[c2] - 1] = c1;
      stencw[c1]++;
      stencw[c2]++;
    }
  }
  for (int c = 1; c <= n_cells; ++c) {
    int lo = row[c - 1] + 1, hi = row[c - 1] + stencw[c] - 1;  // 1-based
    if (hi >= lo) std::sort(col + lo - 1, col + hi);
    for (int p = row[c - 1]; p <= row[c] - 1; ++p)
      if (col[p - 1] == c) dia[c - 1] = p;
    if (col[row[c - 1] - 1] != c) return -2;
  }
  for (int s = 1; s <= n_faces; ++s) {
    int c1 = faces_c[2 * (s - 1)], c2 = faces_c[2 * (s - 1) + 1];
    if (c2 > 0) {
      for (int c = row[c1 - 1]; c <= row[c1] - 1; ++c)
        if (col[c - 1] == c2) pos[2 * (s - 1)] = c;
      for (int c = row[c2 - 1]; c <= row[c2] - 1; ++c)
        if (col[c - 1] == c1) pos[2 * (s - 1) + 1] = c;
    }
  }
  return n;
}

// Create_Matrix.f90:148-155
void tfo_face_coef(int n_faces, const double* sx, const double* sy,
                   const double* sz, const double* dx, const double* dy,
                   const double* dz, double* fc) {
  for (int s = 0; s < n_faces; ++s)
    fc[s] = (sx[s] * sx[s] + sy[s] * sy[s] + sz[s] * sz[s]) /
            (dx[s] * sx[s] + dy[s] * sy[s] + dz[s] * sz[s]);
}

// Pressure matrix, Rhie_And_Chow.f90:199-204 for interior faces and
// Compute_Pressure.f90:154-158 for pressure/ambient boundary faces
// (bnd_open[s] != 0).  val must be zeroed by the caller (Compute_Pressure.f90:122).
void tfo_assemble_pressure(int n_faces, const int* faces_c, const int* dia,
                           const int* pos, const double* fc, const double* fw,
                           const double* v_m /* v_m(1..n_cells) */,
                           const int* bnd_open, double* val) {
  // Rhie_And_Chow.f90:183-205: interior faces
  for (int s = 1; s <= n_faces; ++s) {
    int c1 = faces_c[2 * (s - 1)], c2 = faces_c[2 * (s - 1) + 1];
    if (c2 > 0) {
      double fs = fw[s - 1];
      double a12 = fc[s - 1] * (fs * v_m[c1 - 1] + (1.0 - fs) * v_m[c2 - 1]);
      val[pos[2 * (s - 1)] - 1] = -a12;
      val[pos[2 * (s - 1) + 1] - 1] = -a12;
      val[dia[c1 - 1] - 1] = val[dia[c1 - 1] - 1] + a12;
      val[dia[c2 - 1] - 1] = val[dia[c2 - 1] - 1] + a12;
    }
  }
  // Compute_Pressure.f90:140-160: pressure / ambient boundary faces
  for (int s = 1; s <= n_faces; ++s) {
    int c1 = faces_c[2 * (s - 1)], c2 = faces_c[2 * (s - 1) + 1];
    if (c2 <= 0 && bnd_open && bnd_open[s - 1]) {
      double a12 = fc[s - 1] * v_m[c1 - 1];
      val[dia[c1 - 1] - 1] = val[dia[c1 - 1] - 1] + a12;
    }
  }
}

// Momentum matrix with the upwind-blended convection of
// Compute_Momentum.f90:270-297 (ui % blend_matrix true), wall faces adding
// m12 to the diagonal, then Inertial_Term.f90 (LINEAR): diag += rho*vol/dt.
// rho is taken constant.  val must be zeroed by the caller (:196).
void tfo_assemble_momentum(int n_cells, int n_faces, const int* faces_c,
                           const int* dia, const int* pos, const double* fc,
                           const double* flux, const int* bnd_wall,
                           double vis, double rho, const double* vol,
                           double dt, double* val) {
  for (int s = 1; s <= n_faces; ++s) {
    int c1 = faces_c[2 * (s - 1)], c2 = faces_c[2 * (s - 1) + 1];
    double m0 = vis * fc[s - 1];
    double m12 = m0, m21 = m0;
    double f = flux[s - 1];
    m12 = m12 - fmin_f(f, 0.0) * rho;
    m21 = m21 + fmax_f(f, 0.0) * rho;
    if (c2 > 0) {
      val[pos[2 * (s - 1)] - 1] = val[pos[2 * (s - 1)] - 1] - m12;
      val[dia[c1 - 1] - 1] = val[dia[c1 - 1] - 1] + m12;
      val[pos[2 * (s - 1) + 1] - 1] = val[pos[2 * (s - 1) + 1] - 1] - m21;
      val[dia[c2 - 1] - 1] = val[dia[c2 - 1] - 1] + m21;
    } else if (c2 < 0 && bnd_wall && bnd_wall[s - 1]) {
      val[dia[c1 - 1] - 1] = val[dia[c1 - 1] - 1] + m12;
    }
  }
  for (int c = 1; c <= n_cells; ++c) {
    double a0 = rho * vol[c - 1] / dt;
    val[dia[c - 1] - 1] = val[dia[c - 1] - 1] + a0;
  }
}

}  // extern "C"
