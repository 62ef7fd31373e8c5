// refio.cu -- the reference's files: mpDPFT.input, mpDPFT_V.dat,
// mpDPFT_Den.dat, and the InterpolVQ restart from a V file of another grid.
//
// The reference reads its 47-line input with one istringstream per line
// (GetInputParameters, mpDPFT.cpp:633-690), writes the converged fields as
// text (ExportData, mpDPFT.cpp:12492-12519) and restarts from a V file by
// trilinear interpolation onto the new lattice (LoadV, mpDPFT.cpp:6445-6499).
// Parsing and formatting are host code; the interpolation runs on the GPU.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpdpft_gpu.h"
#include "engine.h"

namespace mpdpft {

namespace {

// Leading numeric tokens of a line, as `iss >> val` reads them: the first
// token that is not a number ends the line (the reference's comments start
// with "//").
std::vector<double> numbers(const std::string& line) {
  std::vector<double> v;
  const char* p = line.c_str();
  for (;;) {
    while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
    if (!*p) break;
    char* end = nullptr;
    errno = 0;
    const double x = std::strtod(p, &end);
    if (end == p || (*end && *end != ' ' && *end != '\t' && *end != '\r')) break;
    v.push_back(x);
    p = end;
  }
  return v;
}

bool read_lines(const char* path, std::vector<std::string>& out) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  std::string cur;
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof(buf), f)) > 0) {
    for (size_t i = 0; i < got; ++i) {
      if (buf[i] == '\n') {
        out.push_back(cur);
        cur.clear();
      } else {
        cur.push_back(buf[i]);
      }
    }
  }
  if (!cur.empty()) out.push_back(cur);
  std::fclose(f);
  return true;
}

int need(const std::vector<double>& v, size_t count, int line, const char* name) {
  if (v.size() < count)
    return set_error(MPDPFT_ERR_ARG, "mpDPFT.input line " + std::to_string(line) + " (" + name + "): expected " +
                                         std::to_string(count) + " value(s), found " + std::to_string(v.size()));
  return MPDPFT_OK;
}

template <typename T>
int copy_vec(const std::vector<double>& v, T* dst, int cap, int* n, int line, const char* name) {
  if ((int)v.size() > cap)
    return set_error(MPDPFT_ERR_ARG, "mpDPFT.input line " + std::to_string(line) + " (" + name + "): more than " +
                                         std::to_string(cap) + " values");
  for (size_t i = 0; i < v.size(); ++i) dst[i] = (T)v[i];
  if (n) *n = (int)v.size();
  return MPDPFT_OK;
}

}  // namespace

// ------------------------------------------------------------ mpDPFT.input --
int read_input(const char* path, mpdpft_input* in) {
  std::vector<std::string> lines;
  if (!path || !read_lines(path, lines)) return set_error(MPDPFT_ERR_ARG, std::string("cannot read ") + (path ? path : "(null)"));
  std::memset(in, 0, sizeof(*in));
  if (lines.size() < 47)
    return set_error(MPDPFT_ERR_ARG, "mpDPFT.input has " + std::to_string(lines.size()) + " lines, expected 47");
  in->lines = (int)lines.size();
  std::vector<std::vector<double>> L(47);
  for (int i = 0; i < 47; ++i) L[i] = numbers(lines[i]);
  int st;
  // scalar lines: the first value
  auto I = [&](int line, const char* name, int* dst) -> int {
    if ((st = need(L[line], 1, line, name))) return st;
    *dst = (int)L[line][0];
    return MPDPFT_OK;
  };
  auto D = [&](int line, const char* name, double* dst) -> int {
    if ((st = need(L[line], 1, line, name))) return st;
    *dst = L[line][0];
    return MPDPFT_OK;
  };
  if ((st = I(0, "System", &in->system)) || (st = I(1, "Symmetry", &in->symmetry)) ||
      (st = I(2, "TaskType", &in->task_type)) || (st = I(3, "TaskParameterCount", &in->task_parameter_count)))
    return st;
  if ((st = copy_vec(L[4], in->task_hyperbox, MPDPFT_INPUT_MAX_VEC, &in->n_task_hyperbox, 4, "TaskHyperBox")))
    return st;
  if ((st = I(5, "DIM", &in->dim)) || (st = I(6, "Units", &in->units)) || (st = D(7, "edge", &in->edge)) ||
      (st = I(8, "steps", &in->steps)) || (st = I(9, "S", &in->species)))
    return st;
  if (in->species < 1 || in->species > MPDPFT_MAX_SPECIES)
    return set_error(MPDPFT_ERR_ARG, "mpDPFT.input line 9 (S): " + std::to_string(in->species) +
                                         " species, the engine takes 1 to " + std::to_string(MPDPFT_MAX_SPECIES));
  const int S = in->species;
  auto V = [&](int line, const char* name, double* dst) -> int {  // S-component vectors
    if ((st = need(L[line], S, line, name))) return st;
    for (int s = 0; s < S; ++s) dst[s] = L[line][s];
    return MPDPFT_OK;
  };
  if ((st = V(10, "Abundances", in->abundances)) || (st = D(11, "RelAcc", &in->rel_acc)) ||
      (st = D(12, "InternalAcc", &in->internal_acc)) || (st = I(13, "K", &in->k_resources)) ||
      (st = I(15, "DensityExpression", &in->density_expression)))
    return st;
  if ((st = copy_vec(L[16], in->mpp, MPDPFT_INPUT_MAX_VEC, &in->n_mpp, 16, "mpp")) ||
      (st = copy_vec(L[17], in->Mpp, MPDPFT_INPUT_MAX_VEC, &in->n_Mpp, 17, "Mpp")))
    return st;
  if ((st = V(18, "tauVec", in->tau)) || (st = V(19, "tVec", in->territory)) || (st = V(20, "TVec", in->temperature)))
    return st;
  if ((st = need(L[21], S, 21, "Environments"))) return st;
  for (int s = 0; s < S; ++s) in->environments[s] = (int)L[21][s];
  if ((st = D(22, "stretchfactor", &in->stretchfactor)) || (st = D(23, "Wall", &in->wall)) ||
      (st = D(24, "Noise", &in->noise)) || (st = I(25, "InterpolVQ", &in->interpol_vq)))
    return st;
  if ((st = copy_vec(L[26], in->interactions, MPDPFT_INPUT_MAX_VEC, &in->n_interactions, 26, "Interactions")))
    return st;
  if ((st = D(27, "incrementalV", &in->incremental_v)) || (st = V(28, "muVec", in->mu)) ||
      (st = D(29, "DeltamuModifier", &in->deltamu_modifier)))
    return st;
  if ((st = need(L[30], 3, 30, "Mixer"))) return st;
  for (int i = 0; i < 3; ++i) in->mixer[i] = L[30][i];
  if ((st = V(31, "thetaVec", in->theta)) || (st = D(32, "SCcriterion", &in->sc_criterion)) ||
      (st = I(33, "maxSCcount", &in->max_sc_count)) || (st = I(34, "method", &in->method)) ||
      (st = I(35, "DelFieldMethod", &in->delfield_method)) || (st = I(36, "MovieQ", &in->movie)))
    return st;
  if ((st = copy_vec(L[37], in->schedule, MPDPFT_INPUT_MAX_VEC, &in->n_schedule, 37, "Schedule")) ||
      (st = copy_vec(L[38], in->ekin_types, MPDPFT_INPUT_MAX_VEC, &in->n_ekin_types, 38, "EkinTypes")))
    return st;
  if ((st = D(39, "alpha", &in->alpha)) || (st = D(40, "beta", &in->beta)) || (st = D(41, "gamma", &in->gamma)) ||
      (st = D(42, "gammaH", &in->gamma_h)) || (st = D(43, "degeneracy", &in->degeneracy)))
    return st;
  if ((st = copy_vec(L[44], in->regularize, MPDPFT_INPUT_MAX_VEC, &in->n_regularize, 44, "regularize"))) return st;
  if ((st = D(45, "RegularizationThreshold", &in->regularization_threshold)) || (st = I(46, "Print", &in->print)))
    return st;
  return MPDPFT_OK;
}

static int reject(int line, const char* name, const std::string& why) {
  return set_error(MPDPFT_ERR_ARG, "mpDPFT.input line " + std::to_string(line) + " (" + name + "): " + why);
}

int params_from_input(const mpdpft_input* in, mpdpft_params* p) {
  mpdpft_params_default(p);
  if (in->units != 1) return reject(6, "Units", "only 1 (HO / atomic units) is implemented");
  if (in->dim != 2 && in->dim != 3) return reject(5, "DIM", "the engine computes 2D and 3D grids");
  const int de = in->density_expression;
  if (de != 1 && de != 2 && de != 5 && de != 7)
    return reject(15, "DensityExpression", std::to_string(de) + " is not implemented (1, 2, 5, 7 are)");
  if (in->method != 1) return reject(34, "method", "only 1 (Riemann) is implemented");
  if (de == 5 && in->delfield_method != 5) return reject(35, "DelFieldMethod", "DensityExpression 5 needs method 5");
  const int mixer = (int)(in->mixer[0] + 0.5);
  if (mixer != 0 && mixer != 1) return reject(30, "Mixer", "mode 2 (Pulay2) is not implemented");
  if (in->n_schedule > 1) return reject(37, "Schedule", "one schedule at a time");
  const int sched = in->n_schedule ? in->schedule[0] : 0;
  if (sched != 0 && sched != 5 && sched != 9) return reject(37, "Schedule", std::to_string(sched) + " is not implemented");
  if (in->n_interactions > MPDPFT_MAX_INTERACTIONS) return reject(26, "Interactions", "too many entries");
  p->dim = in->dim;
  p->steps = in->steps;
  p->species = in->species;
  p->edge = in->edge;
  p->rel_acc = in->rel_acc;
  p->density_expression = de;
  int n = 0;
  for (int a = 0; a < in->n_interactions; ++a) {
    const int t = in->interactions[a];
    if (t == 0) continue;  // noninteracting
    if (t != 1 && t != 8 && t != 10 && t != 11 && t != 21)
      return reject(26, "Interactions", "type " + std::to_string(t) + " is not implemented (1, 8, 10, 11, 21 are)");
    p->interactions[n++] = t;
  }
  p->n_interactions = n;
  for (int s = 0; s < in->species; ++s) {
    p->abundances[s] = in->abundances[s];
    p->tau[s] = in->tau[s];
    p->temperature[s] = in->temperature[s];
    p->mu[s] = in->mu[s];
    p->theta[s] = in->theta[s];
  }
  p->incremental_v = in->incremental_v;
  p->deltamu_modifier = in->deltamu_modifier;
  p->mixer = mixer;
  p->pulay_scope = mixer ? (int)(in->mixer[1] + 0.5) : 1;
  if (mixer && (p->pulay_scope < 1 || p->pulay_scope > MPDPFT_MAX_PULAY))
    return reject(30, "Mixer", "Pulay scope must be 1 to " + std::to_string(MPDPFT_MAX_PULAY));
  p->sc_criterion = in->sc_criterion;
  p->max_sc_count = in->max_sc_count;
  p->schedule = sched;
  p->beta = in->beta;
  p->gamma_h = in->gamma_h;
  p->degeneracy = in->degeneracy;
  p->regularization_threshold = in->regularization_threshold;
  p->internal_acc = in->internal_acc;
  if (de == 5) {
    // getDenEnAt: Mpp = {BoolePairs, maxIter, threshold of ar} (mpDPFT.cpp:3366, 3376, 3554)
    if (in->n_Mpp < 3) return reject(17, "Mpp", "DensityExpression 5 needs BoolePairs, maxIter and the Airy threshold");
    p->boole_pairs = (int)in->Mpp[0];
    p->boole_max_iter = (int)(in->Mpp[1] + 0.5);
    p->airy_threshold = std::fabs(in->Mpp[2]);
    if (p->boole_pairs < 1) return reject(17, "Mpp", "BoolePairs must be at least 1");
    if (in->dim == 3) {
      p->gradient_form = MPDPFT_GRADIENT_FINITE_T;
    } else if (p->airy_threshold < 1.0e300) {
      return reject(17, "Mpp", "the 2D Airy-averaged branch (mpDPFT.cpp:3389-3418) is not implemented: set Mpp[2] "
                               "to 1e300 or more for the small-gradient branch everywhere");
    }
  }
  return MPDPFT_OK;
}

}  // namespace mpdpft

namespace mpdpft {

// ------------------------------------------------------ field text files --
static void fmt16(std::string& out, double v) {
  char b[40];
  const int k = std::snprintf(b, sizeof(b), "%.16g", v);
  out.append(b, (size_t)k);
}

int write_field_files(Ctx& c, const char* v_path, const char* den_path) {
  const int S = c.S, dim = c.P.dim, el = c.P.steps + 1;
  const long m = c.n_ref;
  std::vector<std::vector<double>> V(S), N(S);
  int st;
  for (int s = 0; s < S; ++s) {
    V[s].resize(m);
    N[s].resize(m);
    if ((st = c.get_field(MPDPFT_FIELD_POTENTIAL, s, V[s].data(), MPDPFT_LAYOUT_REFERENCE, MPDPFT_MEM_HOST))) return st;
    if ((st = c.get_field(MPDPFT_FIELD_DENSITY, s, N[s].data(), MPDPFT_LAYOUT_REFERENCE, MPDPFT_MEM_HOST))) return st;
  }
  const double x0 = -0.5 * c.P.edge, dx = c.P.edge / c.P.steps;
  if (v_path) {
    FILE* f = std::fopen(v_path, "wb");
    if (!f) return set_error(MPDPFT_ERR_ARG, std::string("cannot write ") + v_path);
    std::string line;
    for (long q = 0; q < m; ++q) {
      line.clear();
      // VecAt: lattice coordinates of the stored point, x slowest (mpDPFT.cpp:7215-7241)
      const long k = q % el, t = q / el;
      const long idx[3] = {dim == 3 ? t / el : t, dim == 3 ? t % el : k, k};
      for (int d = 0; d < dim; ++d) { fmt16(line, x0 + dx * (double)idx[d]); line.push_back(' '); }
      for (int s = 0; s < S; ++s) { fmt16(line, V[s][q]); line.push_back(' '); }
      line.push_back('\n');
      std::fwrite(line.data(), 1, line.size(), f);
    }
    if (std::fclose(f) != 0) return set_error(MPDPFT_ERR_ARG, std::string("write failed: ") + v_path);
  }
  if (den_path) {
    FILE* f = std::fopen(den_path, "wb");
    if (!f) return set_error(MPDPFT_ERR_ARG, std::string("cannot write ") + den_path);
    std::string line;
    for (long q = 0; q < m; ++q) {
      line.clear();
      for (int s = 0; s < S; ++s) {
        fmt16(line, N[s][q]);
        line.push_back(s == S - 1 ? '\n' : ' ');
      }
      std::fwrite(line.data(), 1, line.size(), f);
    }
    if (std::fclose(f) != 0) return set_error(MPDPFT_ERR_ARG, std::string("write failed: ") + den_path);
  }
  return MPDPFT_OK;
}

// ------------------------------------------------- InterpolVQ restart (GPU) --
// Index of the cell [a[c], a[c+1]] holding x, clamped to the outermost
// cells (points beyond the file's box continue its boundary cells
// linearly); a ascending, n >= 2.
__device__ __forceinline__ int cell_of(const double* a, int n, double x) {
  int lo = 0, hi = n - 2;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a[mid] <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Trilinear (2D: bilinear) interpolation of the file's S fields F[s][n^D]
// on axes ax[dim][n] at every point of the target grid (el points per
// axis at x0 + i dx), written to out[s][el^D].
__global__ void k_interp_v(const double* __restrict__ ax, int n, int dim, const double* __restrict__ F, int S,
                           double x0, double dx, int el, double* __restrict__ out) {
  const long total = dim == 3 ? (long)el * el * el : (long)el * el;
  const long nn = dim == 3 ? (long)n * n * n : (long)n * n;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const long k = q % el, t = q / el;
    const long id[3] = {dim == 3 ? t / el : t, dim == 3 ? t % el : k, k};
    int c[3];
    double w[3];
    for (int d = 0; d < dim; ++d) {
      const double* a = ax + (long)d * n;
      const double x = x0 + dx * (double)id[d];
      c[d] = cell_of(a, n, x);
      w[d] = (x - a[c[d]]) / (a[c[d] + 1] - a[c[d]]);
    }
    for (int s = 0; s < S; ++s) {
      const double* f = F + (long)s * nn;
      double v;
      if (dim == 3) {
        auto at = [&](int di, int dj, int dk) { return f[((long)(c[0] + di) * n + (c[1] + dj)) * n + (c[2] + dk)]; };
        const double c00 = at(0, 0, 0) * (1.0 - w[2]) + at(0, 0, 1) * w[2];
        const double c01 = at(0, 1, 0) * (1.0 - w[2]) + at(0, 1, 1) * w[2];
        const double c10 = at(1, 0, 0) * (1.0 - w[2]) + at(1, 0, 1) * w[2];
        const double c11 = at(1, 1, 0) * (1.0 - w[2]) + at(1, 1, 1) * w[2];
        v = (c00 * (1.0 - w[1]) + c01 * w[1]) * (1.0 - w[0]) + (c10 * (1.0 - w[1]) + c11 * w[1]) * w[0];
      } else {
        auto at = [&](int di, int dj) { return f[(long)(c[0] + di) * n + (c[1] + dj)]; };
        v = (at(0, 0) * (1.0 - w[1]) + at(0, 1) * w[1]) * (1.0 - w[0]) + (at(1, 0) * (1.0 - w[1]) + at(1, 1) * w[1]) * w[0];
      }
      out[(long)s * total + q] = v;
    }
  }
}

int interpolate_v_file(Ctx& c, const char* path, double* const* v_out, int layout, int mem, int* n_file) {
  if (!path) return set_error(MPDPFT_ERR_ARG, "null path");
  if (!v_out) return set_error(MPDPFT_ERR_ARG, "null output arrays");
  std::vector<std::string> lines;
  if (!read_lines(path, lines)) return set_error(MPDPFT_ERR_ARG, std::string("cannot read ") + path);
  while (!lines.empty() && numbers(lines.back()).empty()) lines.pop_back();
  const int dim = c.P.dim, S = c.S;
  const long L = (long)lines.size();
  const long n = std::lround(std::pow((double)L, 1.0 / dim));
  const long nn = dim == 3 ? n * n * n : n * n;
  if (n < 2 || nn != L)
    return set_error(MPDPFT_ERR_ARG, std::string(path) + ": " + std::to_string(L) + " lines are not n^" +
                                         std::to_string(dim) + " points");
  std::vector<double> ax((size_t)dim * n), F((size_t)S * nn);
  for (long q = 0; q < L; ++q) {
    const std::vector<double> v = numbers(lines[q]);
    if ((int)v.size() != dim + S)
      return set_error(MPDPFT_ERR_ARG, std::string(path) + " line " + std::to_string(q) + ": " +
                                           std::to_string(v.size()) + " values, expected " + std::to_string(dim + S) +
                                           " (coordinates and one V per species)");
    const long k = q % n, t = q / n;
    const long id[3] = {dim == 3 ? t / n : t, dim == 3 ? t % n : k, k};
    for (int d = 0; d < dim; ++d) {
      bool first = true;  // the axis value is read where the other indices are 0
      for (int e = 0; e < dim; ++e)
        if (e != d && id[e] != 0) first = false;
      if (first) ax[(size_t)d * n + id[d]] = v[d];
    }
    for (int s = 0; s < S; ++s) F[(size_t)s * nn + q] = v[dim + s];
  }
  for (int d = 0; d < dim; ++d)
    for (long i = 0; i + 1 < n; ++i)
      if (!(ax[(size_t)d * n + i + 1] > ax[(size_t)d * n + i]))
        return set_error(MPDPFT_ERR_ARG, std::string(path) + ": coordinates of axis " + std::to_string(d) +
                                             " are not increasing");
  if (n_file) *n_file = (int)n;
  const int el = layout == MPDPFT_LAYOUT_REFERENCE ? c.P.steps + 1 : c.P.steps;
  const long total = dim == 3 ? (long)el * el * el : (long)el * el;
  double *d_ax = nullptr, *d_F = nullptr, *d_out = nullptr;
  cudaError_t e = cudaMalloc(&d_ax, sizeof(double) * ax.size());
  if (e == cudaSuccess) e = cudaMalloc(&d_F, sizeof(double) * F.size());
  if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(double) * (size_t)S * total);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_ax, ax.data(), sizeof(double) * ax.size(), cudaMemcpyHostToDevice, c.stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_F, F.data(), sizeof(double) * F.size(), cudaMemcpyHostToDevice, c.stream);
  if (e == cudaSuccess) {
    k_interp_v<<<grid_blocks(total), kThreads, 0, c.stream>>>(d_ax, (int)n, dim, d_F, S, -0.5 * c.P.edge,
                                                             c.P.edge / c.P.steps, el, d_out);
    e = cudaGetLastError();
  }
  for (int s = 0; s < S && e == cudaSuccess; ++s) {
    if (!v_out[s]) continue;
    e = cudaMemcpyAsync(v_out[s], d_out + (size_t)s * total, sizeof(double) * total,
                        mem == MPDPFT_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, c.stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
  cudaFree(d_ax);
  cudaFree(d_F);
  cudaFree(d_out);
  if (e != cudaSuccess) return set_error(MPDPFT_ERR_CUDA, std::string("interpolate_v_file: ") + cudaGetErrorString(e));
  return MPDPFT_OK;
}

}  // namespace mpdpft

extern "C" {

int mpdpft_read_input(const char* path, mpdpft_input* out) {
  if (!out) return mpdpft::set_error(MPDPFT_ERR_ARG, "null output");
  return mpdpft::read_input(path, out);
}

int mpdpft_params_from_input(const mpdpft_input* in, mpdpft_params* out) {
  if (!in || !out) return mpdpft::set_error(MPDPFT_ERR_ARG, "null argument");
  return mpdpft::params_from_input(in, out);
}

}  // extern "C"
