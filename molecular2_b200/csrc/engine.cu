// Engine lifetime, basis normalisation, Boys table, basis transforms and the
// C entry points that are not integral kernels.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "engine.h"
#include "md.cuh"

namespace m2 {

int set_error(jk_engine* e, int code, const std::string& msg) {
  if (e) e->err = msg;
  return code;
}

int check_cuda(jk_engine* e, cudaError_t st, const char* what) {
  if (st == cudaSuccess) return JK_OK;
  int code = (st == cudaErrorMemoryAllocation) ? JK_ERR_NOMEM : JK_ERR_CUDA;
  return set_error(e, code, std::string(what) + ": " + cudaGetErrorString(st));
}

static double dfact(int n) {
  double r = 1.0;
  for (int k = n; k > 1; k -= 2) r *= k;
  return r;
}

// Normalise as libint2::Shell: primitive norms for x^l, then the contracted
// x^l function to unit norm.
static void normalise_shell(int l, const double* a, double* c, int np) {
  for (int p = 0; p < np; ++p)
    c[p] *= std::sqrt(std::pow(4.0 * a[p], l) * std::pow(2.0 * a[p] / M_PI, 1.5) / dfact(2 * l - 1));
  double s = 0.0;
  for (int p = 0; p < np; ++p)
    for (int q = 0; q < np; ++q) {
      double g = a[p] + a[q];
      s += c[p] * c[q] * dfact(2 * l - 1) / std::pow(2.0 * g, l) * std::pow(M_PI / g, 1.5);
    }
  s = 1.0 / std::sqrt(s);
  for (int p = 0; p < np; ++p) c[p] *= s;
}

int build_basis(const jk_basis* b, bool allow_pure, int lmax, HostBasis& out, std::string& err) {
  if (!b || b->nshell <= 0 || !b->l || !b->nprim || !b->prim_off || !b->exps || !b->coefs || !b->xyz) {
    err = "basis: null array or empty basis";
    return JK_ERR_ARG;
  }
  HostBasis h;
  h.nshell = b->nshell;
  h.off_final.push_back(0);
  h.off_cart.push_back(0);
  for (int s = 0; s < b->nshell; ++s) {
    int l = b->l[s];
    if (l < 0 || l > lmax) {
      err = "basis: shell " + std::to_string(s) + " has l=" + std::to_string(l) + " (supported up to " +
            std::to_string(lmax) + ")";
      return JK_ERR_ARG;
    }
    int np = b->nprim[s];
    if (np <= 0) {
      err = "basis: shell " + std::to_string(s) + " has no primitives";
      return JK_ERR_ARG;
    }
    int pure = (allow_pure && b->pure && b->pure[s] && l >= 2) ? 1 : 0;
    h.l.push_back(l);
    h.nprim.push_back(np);
    h.prim_off.push_back((int)h.exps.size());
    h.pure.push_back(pure);
    h.atom.push_back(b->atom ? b->atom[s] : -1);
    for (int i = 0; i < 3; ++i) h.xyz.push_back(b->xyz[3 * s + i]);
    std::vector<double> a(b->exps + b->prim_off[s], b->exps + b->prim_off[s] + np);
    std::vector<double> c(b->coefs + b->prim_off[s], b->coefs + b->prim_off[s] + np);
    for (double x : a)
      if (!(x > 0.0)) {
        err = "basis: shell " + std::to_string(s) + " has a non-positive exponent";
        return JK_ERR_ARG;
      }
    normalise_shell(l, a.data(), c.data(), np);
    h.exps.insert(h.exps.end(), a.begin(), a.end());
    h.coefs.insert(h.coefs.end(), c.begin(), c.end());
    h.off_final.push_back(h.off_final.back() + (pure ? 2 * l + 1 : ncart(l)));
    h.off_cart.push_back(h.off_cart.back() + ncart(l));
    h.max_l = std::max(h.max_l, l);
  }
  h.n_final = h.off_final.back();
  h.n_cart = h.off_cart.back();
  out = std::move(h);
  return JK_OK;
}

// Real solid harmonics (rows m=-l..l) over x^l-normalised Cartesian
// components, built from the Cartesian recursion for regular solid harmonics
// (Helgaker, Jorgensen & Olsen eqs. 6.4.70-6.4.73) and normalised in the
// metric of the Cartesian functions.
static std::vector<double> solid_harmonic_block(int l) {
  const int D = l + 3;  // exponent box
  auto id = [&](int a, int b, int c) { return (a * D + b) * D + c; };
  std::vector<std::vector<std::vector<double>>> S(l + 1);
  S[0].assign(1, std::vector<double>(D * D * D, 0.0));
  S[0][0][id(0, 0, 0)] = 1.0;
  auto addmul = [&](const std::vector<double>& p, int dx, int dy, int dz, double f, std::vector<double>& o) {
    for (int a = 0; a < D; ++a)
      for (int b = 0; b < D; ++b)
        for (int c = 0; c < D; ++c) {
          double v = p[id(a, b, c)];
          if (v != 0.0 && a + dx < D && b + dy < D && c + dz < D) o[id(a + dx, b + dy, c + dz)] += f * v;
        }
  };
  for (int k = 0; k < l; ++k) {
    S[k + 1].assign(2 * k + 3, std::vector<double>(D * D * D, 0.0));
    double f = std::sqrt((k == 0 ? 2.0 : 1.0) * (2 * k + 1) / (2.0 * k + 2));
    addmul(S[k][2 * k], 1, 0, 0, f, S[k + 1][2 * k + 2]);
    if (k > 0) addmul(S[k][0], 0, 1, 0, -f, S[k + 1][2 * k + 2]);
    addmul(S[k][2 * k], 0, 1, 0, f, S[k + 1][0]);
    if (k > 0) addmul(S[k][0], 1, 0, 0, f, S[k + 1][0]);
    for (int m = -k; m <= k; ++m) {
      double den = std::sqrt((double)(k + m + 1) * (k - m + 1));
      addmul(S[k][m + k], 0, 0, 1, (2 * k + 1) / den, S[k + 1][m + k + 1]);
      if (k > 0 && std::abs(m) <= k - 1) {
        double g = -std::sqrt((double)(k + m) * (k - m)) / den;
        addmul(S[k - 1][m + k - 1], 2, 0, 0, g, S[k + 1][m + k + 1]);
        addmul(S[k - 1][m + k - 1], 0, 2, 0, g, S[k + 1][m + k + 1]);
        addmul(S[k - 1][m + k - 1], 0, 0, 2, g, S[k + 1][m + k + 1]);
      }
    }
  }
  const int nc = ncart(l);
  std::vector<double> R((2 * l + 1) * nc);
  for (int m = 0; m < 2 * l + 1; ++m) {
    for (int i = 0; i < nc; ++i) R[m * nc + i] = S[l][m][id(cart_a(l, i), cart_b(l, i), cart_c(l, i))];
    double nrm = 0.0;
    for (int i = 0; i < nc; ++i)
      for (int j = 0; j < nc; ++j) {
        int sx = cart_a(l, i) + cart_a(l, j), sy = cart_b(l, i) + cart_b(l, j), sz = cart_c(l, i) + cart_c(l, j);
        if (sx % 2 || sy % 2 || sz % 2) continue;
        nrm += R[m * nc + i] * R[m * nc + j] * dfact(sx - 1) * dfact(sy - 1) * dfact(sz - 1) / dfact(2 * l - 1);
      }
    for (int i = 0; i < nc; ++i) R[m * nc + i] /= std::sqrt(nrm);
  }
  return R;
}

int upload_basis(jk_engine* e, const HostBasis& hb, DevBasis& db) {
  cudaStream_t s = e->stream;
  std::vector<double> x(hb.nshell), y(hb.nshell), z(hb.nshell);
  for (int i = 0; i < hb.nshell; ++i) {
    x[i] = hb.xyz[3 * i];
    y[i] = hb.xyz[3 * i + 1];
    z[i] = hb.xyz[3 * i + 2];
  }
  std::vector<double> sph;
  for (int l = 0; l <= SPH_LMAX; ++l) {
    auto blk = solid_harmonic_block(l);
    sph.insert(sph.end(), blk.begin(), blk.end());
  }
  std::vector<int> cs, cc, fs, fc;
  for (int sh = 0; sh < hb.nshell; ++sh) {
    for (int i = 0; i < ncart(hb.l[sh]); ++i) {
      cs.push_back(sh);
      cc.push_back(i);
    }
    for (int i = 0; i < hb.off_final[sh + 1] - hb.off_final[sh]; ++i) {
      fs.push_back(sh);
      fc.push_back(i);
    }
  }
  cudaError_t st = cudaSuccess;
#define UP(buf, vec) \
  if (st == cudaSuccess) st = buf.upload(vec, s)
  UP(db.l, hb.l);
  UP(db.cart_off, hb.off_cart);
  UP(db.final_off, hb.off_final);
  UP(db.nprim, hb.nprim);
  UP(db.prim_off, hb.prim_off);
  UP(db.atom, hb.atom);
  UP(db.pure, hb.pure);
  UP(db.x, x);
  UP(db.y, y);
  UP(db.z, z);
  UP(db.exps, hb.exps);
  UP(db.coefs, hb.coefs);
  UP(db.sph, sph);
  UP(db.cart_shell, cs);
  UP(db.cart_comp, cc);
  UP(db.final_shell, fs);
  UP(db.final_comp, fc);
#undef UP
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);  // host vectors die on return
  return check_cuda(e, st, "upload basis");
}

// Boys table: F_m(k h), m < BOYS_NCOL, by the convergent series at the top
// order and downward recursion.
static std::vector<double> boys_table() {
  std::vector<double> t(BOYS_NGRID * BOYS_NCOL);
  const int M = BOYS_NCOL - 1;
  for (int k = 0; k < BOYS_NGRID; ++k) {
    double T = k * BOYS_STEP;
    double term = 1.0 / (2 * M + 1), sum = term;
    for (int j = 1; j < 2000; ++j) {
      term *= 2.0 * T / (2 * M + 2 * j + 1);
      sum += term;
      if (term < 1e-18 * sum) break;
    }
    double ex = std::exp(-T);
    double* row = &t[k * BOYS_NCOL];
    row[M] = ex * sum;
    for (int m = M - 1; m >= 0; --m) row[m] = (2.0 * T * row[m + 1] + ex) / (2 * m + 1);
  }
  return t;
}

// ---------------------------------------------------------------- transforms
// Dc[a][b] = sum T[mu][a] Df[mu][nu] T[nu][b] over the shells' pure blocks
// (identity for Cartesian shells).  One thread per Cartesian element.
__global__ void k_final_to_cart(int nc, int n, const int* __restrict__ cshell, const int* __restrict__ ccomp,
                                const int* __restrict__ l, const int* __restrict__ pure,
                                const int* __restrict__ foff, const double* __restrict__ sph,
                                const double* __restrict__ Df, double* __restrict__ Dc) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = blockIdx.y;
  if (b >= nc) return;
  const int sa = cshell[a], sb = cshell[b], ia = ccomp[a], ib = ccomp[b];
  const int la = l[sa], lb = l[sb], fa = foff[sa], fb = foff[sb];
  const int pa = pure[sa], pb = pure[sb];
  const int na = pa ? 2 * la + 1 : 1, nb = pb ? 2 * lb + 1 : 1;
  double v = 0.0;
  for (int m = 0; m < na; ++m) {
    const double ta = pa ? sph[sph_off(la) + m * ncart(la) + ia] : 1.0;
    if (ta == 0.0) continue;
    const int fm = pa ? fa + m : fa + ia;
    for (int k = 0; k < nb; ++k) {
      const double tb = pb ? sph[sph_off(lb) + k * ncart(lb) + ib] : 1.0;
      const int fk = pb ? fb + k : fb + ib;
      v += ta * tb * Df[(size_t)fk * n + fm];
    }
  }
  Dc[(size_t)b * nc + a] = v;
}

// Xf[mu][nu] = scale * sum T[mu][a] (Xc[a][b] + Xc[b][a]) T[nu][b].
__global__ void k_cart_to_final_sym(int nc, int n, const int* __restrict__ fshell, const int* __restrict__ fcomp,
                                    const int* __restrict__ l, const int* __restrict__ pure,
                                    const int* __restrict__ coff, const double* __restrict__ sph,
                                    const double* __restrict__ Xc, double scale, double* __restrict__ Xf) {
  const int nu = blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  if (nu >= n) return;
  const int sa = fshell[mu], sb = fshell[nu], im = fcomp[mu], in = fcomp[nu];
  const int la = l[sa], lb = l[sb], ca = coff[sa], cb = coff[sb];
  const int pa = pure[sa], pb = pure[sb];
  const int na = pa ? ncart(la) : 1, nb = pb ? ncart(lb) : 1;
  double v = 0.0;
  for (int i = 0; i < na; ++i) {
    const double ta = pa ? sph[sph_off(la) + im * ncart(la) + i] : 1.0;
    if (ta == 0.0) continue;
    const int a = pa ? ca + i : ca + im;
    for (int j = 0; j < nb; ++j) {
      const double tb = pb ? sph[sph_off(lb) + in * ncart(lb) + j] : 1.0;
      const int b = pb ? cb + j : cb + in;
      v += ta * tb * (Xc[(size_t)b * nc + a] + Xc[(size_t)a * nc + b]);
    }
  }
  Xf[(size_t)nu * n + mu] = scale * v;
}

// Dn[s1][s2] = max |Df| over the shell block (Eigen lpNorm<Infinity>), and
// the global maximum in *Dmax (non-negative doubles order like their bits).
__global__ void k_shell_norms(int nshell, int n, const int* __restrict__ foff, const double* __restrict__ Df,
                              double* __restrict__ Dn, unsigned long long* __restrict__ Dmax) {
  const int s2 = blockIdx.x * blockDim.x + threadIdx.x;
  const int s1 = blockIdx.y;
  if (s2 >= nshell) return;
  double m = 0.0;
  for (int i = foff[s1]; i < foff[s1 + 1]; ++i)
    for (int j = foff[s2]; j < foff[s2 + 1]; ++j) m = fmax(m, fabs(Df[(size_t)j * n + i]));
  Dn[(size_t)s1 * nshell + s2] = m;
  atomicMax(Dmax, (unsigned long long)__double_as_longlong(m));
}

void launch_final_to_cart(const jk_engine* e, const double* Dfinal, double* Dcart, cudaStream_t s) {
  const int nc = e->obs.n_cart, n = e->obs.n_final;
  dim3 grid((nc + 127) / 128, nc);
  k_final_to_cart<<<grid, 128, 0, s>>>(nc, n, e->dobs.cart_shell.p, e->dobs.cart_comp.p, e->dobs.l.p,
                                       e->dobs.pure.p, e->dobs.final_off.p, e->dobs.sph.p, Dfinal, Dcart);
}

void launch_cart_to_final_sym(const jk_engine* e, const double* Xcart, double scale, double* Xfinal,
                              cudaStream_t s) {
  const int nc = e->obs.n_cart, n = e->obs.n_final;
  dim3 grid((n + 127) / 128, n);
  k_cart_to_final_sym<<<grid, 128, 0, s>>>(nc, n, e->dobs.final_shell.p, e->dobs.final_comp.p, e->dobs.l.p,
                                           e->dobs.pure.p, e->dobs.cart_off.p, e->dobs.sph.p, Xcart, scale,
                                           Xfinal);
}

__global__ void k_add(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ c, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) c[i] = a[i] + b[i];
}

void launch_add(const double* a, const double* b, double* c, size_t n, cudaStream_t s) {
  k_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, c, n);
}

void launch_shell_norms(const jk_engine* e, const double* Dfinal, double* Dnorm, double* Dmax, cudaStream_t s) {
  const int ns = e->obs.nshell, n = e->obs.n_final;
  cudaMemsetAsync(Dmax, 0, sizeof(double), s);
  dim3 grid((ns + 127) / 128, ns);
  k_shell_norms<<<grid, 128, 0, s>>>(ns, n, e->dobs.final_off.p, Dfinal, Dnorm, (unsigned long long*)Dmax);
}

}  // namespace m2

using namespace m2;

extern "C" {

int jk_create(const jk_basis* obs, const jk_basis* aux, int natom, const double* atom_xyz, const double* Z,
              int device, jk_engine** out) {
  if (!out) return JK_ERR_ARG;
  *out = nullptr;
  jk_engine* e = new (std::nothrow) jk_engine();
  if (!e) return JK_ERR_NOMEM;
  int rc = JK_OK;
  std::string err;
  if (natom < 0 || (natom > 0 && (!atom_xyz || !Z))) {
    rc = JK_ERR_ARG;
    err = "jk_create: atoms";
  }
  if (rc == JK_OK) rc = build_basis(obs, true, MAX_L_OBS, e->obs, err);
  if (rc == JK_OK && aux) {
    rc = build_basis(aux, true, MAX_L_AUX, e->aux, err);
    e->has_aux = (rc == JK_OK);
  }
  if (rc != JK_OK) {
    // keep the message reachable: hand back the engine in an error state
    e->err = err;
    *out = e;
    return rc;
  }
  e->natom = natom;
  e->atom_xyz.assign(atom_xyz, atom_xyz + 3 * natom);
  e->Z.assign(Z, Z + natom);
  e->device = device;
  cudaError_t st = cudaSetDevice(device);
  if (st == cudaSuccess) st = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
  for (int i = 0; i < jk_engine::NCLS_STREAMS && st == cudaSuccess; ++i) {
    st = cudaStreamCreateWithFlags(&e->cls_stream[i], cudaStreamNonBlocking);
    if (st == cudaSuccess) st = cudaEventCreateWithFlags(&e->cls_join[i], cudaEventDisableTiming);
  }
  if (st == cudaSuccess) st = cudaEventCreateWithFlags(&e->cls_fork, cudaEventDisableTiming);
  if (st != cudaSuccess) {
    rc = check_cuda(e, st, "jk_create: device/stream");
    *out = e;
    return rc;
  }
  if (cublasCreate(&e->cublas) != CUBLAS_STATUS_SUCCESS ||
      cublasSetStream(e->cublas, e->stream) != CUBLAS_STATUS_SUCCESS) {
    *out = e;
    return set_error(e, JK_ERR_CUDA, "jk_create: cublasCreate failed");
  }
  if (cusolverDnCreate(&e->cusolver) != CUSOLVER_STATUS_SUCCESS ||
      cusolverDnSetStream(e->cusolver, e->stream) != CUSOLVER_STATUS_SUCCESS) {
    *out = e;
    return set_error(e, JK_ERR_CUDA, "jk_create: cusolverDnCreate failed");
  }
  rc = upload_basis(e, e->obs, e->dobs);
  if (rc == JK_OK && e->has_aux) rc = upload_basis(e, e->aux, e->daux);
  if (rc == JK_OK) rc = check_cuda(e, e->boys.upload(boys_table(), e->stream), "boys table");
  if (rc == JK_OK) rc = check_cuda(e, cudaStreamSynchronize(e->stream), "boys table");
  if (rc == JK_OK) rc = build_pairs(e);
  *out = e;
  return rc;
}

void jk_destroy(jk_engine* e) {
  if (!e) return;
  if (e->stream) cudaStreamSynchronize(e->stream);
  if (e->cublas) cublasDestroy(e->cublas);
  if (e->cusolver) cusolverDnDestroy(e->cusolver);
  for (auto& ev : e->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : e->kev) cudaEventDestroy(ev);
  for (int i = 0; i < jk_engine::NCLS_STREAMS; ++i) {
    if (e->cls_stream[i]) cudaStreamSynchronize(e->cls_stream[i]);
    if (e->cls_stream[i]) cudaStreamDestroy(e->cls_stream[i]);
    if (e->cls_join[i]) cudaEventDestroy(e->cls_join[i]);
  }
  if (e->cls_fork) cudaEventDestroy(e->cls_fork);
  cudaStream_t s = e->stream;
  delete e;  // frees device buffers
  if (s) cudaStreamDestroy(s);
}

const char* jk_last_error(const jk_engine* e) { return e ? e->err.c_str() : "null engine"; }

namespace m2 {
ClassStreams::ClassStreams(jk_engine* e_, cudaStream_t s_) : e(e_), s(s_) {
  cudaEventRecord(e->cls_fork, s);
  for (int i = 0; i < jk_engine::NCLS_STREAMS; ++i) cudaStreamWaitEvent(e->cls_stream[i], e->cls_fork, 0);
}
cudaStream_t ClassStreams::next(double cost) {
  int best = 0;
  for (int i = 1; i < jk_engine::NCLS_STREAMS; ++i)
    if (load[i] < load[best]) best = i;
  load[best] += cost;
  return e->cls_stream[best];
}
void ClassStreams::join() {
  for (int i = 0; i < jk_engine::NCLS_STREAMS; ++i) {
    cudaEventRecord(e->cls_join[i], e->cls_stream[i]);
    cudaStreamWaitEvent(s, e->cls_join[i], 0);
  }
}
}  // namespace m2

int jk_sizes(const jk_engine* e, int* n, int* naux, int* nshell) {
  if (!e) return JK_ERR_ARG;
  if (n) *n = e->obs.n_final;
  if (naux) *naux = e->has_aux ? e->aux.n_final : 0;
  if (nshell) *nshell = e->obs.nshell;
  return JK_OK;
}

int jk_schwarz(const jk_engine* e, double* Q) {
  if (!e || !Q) return JK_ERR_ARG;
  if (e->schwarz_host.empty()) return JK_ERR_STATE;
  std::memcpy(Q, e->schwarz_host.data(), e->schwarz_host.size() * sizeof(double));
  return JK_OK;
}

long long jk_last_quartets(const jk_engine* e) {
  if (!e || !e->last_counter) return -1;
  unsigned long long c = 0;
  if (cudaMemcpyAsync(&c, e->last_counter, sizeof(c), cudaMemcpyDeviceToHost, e->stream) != cudaSuccess) return -1;
  if (cudaStreamSynchronize(e->stream) != cudaSuccess) return -1;
  return (long long)c;
}

}  // extern "C"
