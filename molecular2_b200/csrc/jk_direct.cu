// Integral-direct J/K build (FP64) — the B200 replacement for
// Fock::formJKdirect (molecular2 src/fockbuild.cpp:64-164).
//
// Work decomposition.  Shell pairs (a,b) with l_a >= l_b are grouped into the
// six angular classes ss, ps, pp, ds, dp, dd and, inside a class, sorted by
// their Schwarz bound Q_ab (descending).  A unique shell quartet is a pair of
// pairs {ab, cd}: class(ab) > class(cd), or the same class with index(cd) <=
// index(ab).  One kernel instantiation per class pair (21 for l <= 2), the 21
// launches of a build spread longest first over the engine's side streams so
// that they run concurrently; a block owns one bra pair and a chunk of kets,
// one thread one quartet.  Because kets
// are Q-sorted, the kets that can pass Q_ab Q_cd Dmax >= precision form a
// prefix found by binary search; each quartet then applies molecular2's
// screen max6(|D| shell blocks) Q_ab Q_cd >= precision (:111-115).
//
// Digestion follows :121-153 (6 updates with the permutational degeneracy
// factor, symmetrised at the end with the 1/4 of :161-162).  J_ab is shared by
// the whole block and is reduced with warp shuffles before one atomic per
// element per warp; the other five blocks are accumulated per quartet and
// added with FP64 atomics.  Everything runs in the Cartesian representation:
// D is transformed to Cartesian functions first and J, K back afterwards.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "engine.h"
#include "jk_kernels.cuh"

namespace m2 {

PairView view(const PairClassDev& c) { return PairView{c.sa.p, c.sb.p, c.prim_off.p, c.nprim.p, c.Q.p, c.npair}; }

PrimView prim_view(const jk_engine* e) { return PrimView{e->pp_p.p, e->pp_x.p, e->pp_y.p, e->pp_z.p, e->pp_K.p}; }

ShellView shell_view(const jk_engine* e) {
  return ShellView{e->dobs.x.p, e->dobs.y.p, e->dobs.z.p, e->dobs.cart_off.p};
}

static void launch_schwarz(int la, int lb, const SchwarzParams& P, int npair, cudaStream_t s) {
  dim3 grid((npair + 63) / 64);
  if (la == 0 && lb == 0) k_schwarz<0, 0><<<grid, 64, 0, s>>>(P);
  if (la == 1 && lb == 0) k_schwarz<1, 0><<<grid, 64, 0, s>>>(P);
  if (la == 1 && lb == 1) k_schwarz<1, 1><<<grid, 64, 0, s>>>(P);
  if (la == 2 && lb == 0) k_schwarz<2, 0><<<grid, 64, 0, s>>>(P);
  if (la == 2 && lb == 1) k_schwarz<2, 1><<<grid, 64, 0, s>>>(P);
  if (la == 2 && lb == 2) launch_schwarz_dd(P, grid, s);
}

int build_pairs(jk_engine* e) {
  const HostBasis& hb = e->obs;
  std::vector<PairClassHost> cls(NPAIRCLASS);
  for (int la = 0; la <= MAX_L_OBS; ++la)
    for (int lb = 0; lb <= la; ++lb) {
      cls[pair_class(la, lb)].la = la;
      cls[pair_class(la, lb)].lb = lb;
    }
  std::vector<double> pp_p, pp_x, pp_y, pp_z, pp_K, pp_a;
  for (int i = 0; i < hb.nshell; ++i)
    for (int j = 0; j < hb.nshell; ++j) {
      const int li = hb.l[i], lj = hb.l[j];
      if (li < lj || (li == lj && j > i)) continue;  // canonical orientation l_a >= l_b
      PairClassHost& c = cls[pair_class(li, lj)];
      const double* A = &hb.xyz[3 * i];
      const double* B = &hb.xyz[3 * j];
      const double AB2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
      int off = (int)pp_p.size(), cnt = 0;
      for (int pa = 0; pa < hb.nprim[i]; ++pa)
        for (int pb = 0; pb < hb.nprim[j]; ++pb) {
          const double al = hb.exps[hb.prim_off[i] + pa], be = hb.exps[hb.prim_off[j] + pb];
          const double p = al + be;
          const double K = hb.coefs[hb.prim_off[i] + pa] * hb.coefs[hb.prim_off[j] + pb] * std::exp(-al * be / p * AB2);
          if (std::fabs(K) < 1e-18) continue;  // contributes below 1e-18 Eh to any integral
          pp_p.push_back(p);
          pp_x.push_back((al * A[0] + be * B[0]) / p);
          pp_y.push_back((al * A[1] + be * B[1]) / p);
          pp_z.push_back((al * A[2] + be * B[2]) / p);
          pp_K.push_back(K);
          pp_a.push_back(al);
          ++cnt;
        }
      if (cnt == 0) continue;  // every primitive product vanishes: the pair cannot contribute
      c.sa.push_back(i);
      c.sb.push_back(j);
      c.prim_off.push_back(off);
      c.nprim.push_back(cnt);
    }
  cudaStream_t s = e->stream;
  cudaError_t st = cudaSuccess;
  if (st == cudaSuccess) st = e->pp_p.upload(pp_p, s);
  if (st == cudaSuccess) st = e->pp_x.upload(pp_x, s);
  if (st == cudaSuccess) st = e->pp_y.upload(pp_y, s);
  if (st == cudaSuccess) st = e->pp_z.upload(pp_z, s);
  if (st == cudaSuccess) st = e->pp_K.upload(pp_K, s);
  if (st == cudaSuccess) st = e->pp_a.upload(pp_a, s);
  if (st != cudaSuccess) return check_cuda(e, st, "upload primitive pairs");

  // Schwarz bounds on the GPU, class by class
  const int ns = hb.nshell;
  e->schwarz_host.assign((size_t)ns * ns, 0.0);
  e->Qmax = 0.0;
  for (int k = 0; k < NPAIRCLASS; ++k) {
    PairClassHost& c = cls[k];
    PairClassDev& d = e->pcls[k];
    d.la = c.la;
    d.lb = c.lb;
    d.npair = (int)c.sa.size();
    if (d.npair == 0) continue;
    st = d.sa.upload(c.sa, s);
    if (st == cudaSuccess) st = d.sb.upload(c.sb, s);
    if (st == cudaSuccess) st = d.prim_off.upload(c.prim_off, s);
    if (st == cudaSuccess) st = d.nprim.upload(c.nprim, s);
    if (st == cudaSuccess) st = d.Q.alloc(d.npair);
    if (st != cudaSuccess) return check_cuda(e, st, "upload pairs");
    SchwarzParams P{view(d), prim_view(e), shell_view(e), e->dobs.l.p, e->dobs.pure.p, e->dobs.sph.p,
                    e->boys.p, d.Q.p};
    launch_schwarz(c.la, c.lb, P, d.npair, s);
    c.Q.resize(d.npair);
    st = cudaMemcpyAsync(c.Q.data(), d.Q.p, d.npair * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (st == cudaSuccess) st = cudaStreamSynchronize(s);
    if (st != cudaSuccess) return check_cuda(e, st, "schwarz kernel");
    // sort the class by Q descending
    std::vector<int> order(d.npair);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return c.Q[x] > c.Q[y]; });
    // inside windows of PAIR_WINDOW, longest contractions first (warps of
    // kets with similar primitive counts; kernels round Q prefixes to windows)
    for (size_t w0 = 0; w0 < order.size(); w0 += PAIR_WINDOW) {
      const size_t w1 = std::min(order.size(), w0 + (size_t)PAIR_WINDOW);
      std::stable_sort(order.begin() + w0, order.begin() + w1,
                       [&](int x, int y) { return c.nprim[x] > c.nprim[y]; });
    }
    PairClassHost sorted;
    for (int o : order) {
      sorted.sa.push_back(c.sa[o]);
      sorted.sb.push_back(c.sb[o]);
      sorted.prim_off.push_back(c.prim_off[o]);
      sorted.nprim.push_back(c.nprim[o]);
      sorted.Q.push_back(c.Q[o]);
      e->schwarz_host[(size_t)c.sa[o] * ns + c.sb[o]] = c.Q[o];
      e->schwarz_host[(size_t)c.sb[o] * ns + c.sa[o]] = c.Q[o];
      e->Qmax = std::max(e->Qmax, c.Q[o]);
    }
    st = d.sa.upload(sorted.sa, s);
    if (st == cudaSuccess) st = d.sb.upload(sorted.sb, s);
    if (st == cudaSuccess) st = d.prim_off.upload(sorted.prim_off, s);
    if (st == cudaSuccess) st = d.nprim.upload(sorted.nprim, s);
    if (st == cudaSuccess) st = d.Q.upload(sorted.Q, s);
    if (st == cudaSuccess) st = cudaStreamSynchronize(s);
    if (st != cudaSuccess) return check_cuda(e, st, "upload sorted pairs");
  }
  st = e->schwarz_dev.upload(e->schwarz_host, s);
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);
  return check_cuda(e, st, "schwarz matrix");
}

// Kets per block: one per thread (128) when the class has enough (bra, chunk)
// blocks to fill the GPU; classes with few bra pairs take smaller chunks so
// their work still spreads over about 4 blocks per SM (idle threads of a
// block only cost its residency).
static int ket_chunk(int nbra, int nket_max) {
  int k = 128;
  while (k > 32 && (long long)nbra * ((nket_max + k - 1) / k) < 4 * 148) k /= 2;
  return k;
}

// Rough relative cost of one class launch (Cartesian products of the pair
// classes ss ps pp ds dp dd times the pair counts): orders the launches
// longest first over the side streams.
static double class_cost(int A, int B, int nbra, int nket) {
  static const double ncp[6] = {1, 3, 9, 6, 18, 36};
  return (double)nbra * nket * ncp[A] * ncp[B] * (A == B ? 0.5 : 1.0);
}

// Every (bra class, ket class) launch of one build, longest first, spread over
// the engine's side streams so that the small d classes run beside the large
// ones instead of one after another; J, K and the counters are accumulated
// with atomics, so the launches commute.
template <class Launch>
static void launch_classes(jk_engine* e, cudaStream_t s, Launch&& launch) {
  struct Item {
    int A, B;
    double cost;
  };
  std::vector<Item> items;
  for (int A = 0; A < NPAIRCLASS; ++A)
    for (int B = 0; B <= A; ++B)
      if (e->pcls[A].npair && e->pcls[B].npair)
        items.push_back({A, B, class_cost(A, B, e->pcls[A].npair, e->pcls[B].npair)});
  std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.cost > b.cost; });
  ClassStreams cs(e, s);
  for (const Item& it : items) launch(it.A, it.B, cs.next(it.cost));
  cs.join();
}

static void launch_jk(const jk_engine* e, int A, int B, const JKParams& Pin, int nbra, int nket_max, cudaStream_t s,
                      int nden = 1) {
  JKParams P = Pin;
  int nb = 0;
  bra_share(e, nbra, P.bra0, P.bra_step, nb);
  if (nb == 0) return;
  P.kchunk = ket_chunk(nb, nket_max);
  dim3 grid(nb, (nket_max + P.kchunk - 1) / P.kchunk);
  if (A <= 2)
    launch_jk_bra_s(A, B, nden, P, grid, s);
  else if (A == 3)
    launch_jk_bra_ds(B, nden, P, grid, s);
  else if (A == 4)
    launch_jk_bra_dp(B, nden, P, grid, s);
  else if (B < 4)
    launch_jk_bra_dd_lo(B, nden, P, grid, s);
  else
    launch_jk_bra_dd_hi(B, nden, P, grid, s);
}

int direct_jk_device(jk_engine* e, const double* dD, double precision, double mult, double* dJ, double* dK,
                     cudaStream_t s) {
  const int nc = e->obs.n_cart, ns = e->obs.nshell;
  cudaError_t st = cudaSuccess;
  if (st == cudaSuccess) st = e->Dcart.alloc((size_t)nc * nc);
  if (st == cudaSuccess) st = e->Jcart.alloc((size_t)nc * nc);
  if (st == cudaSuccess) st = e->Kcart.alloc((size_t)nc * nc);
  if (st == cudaSuccess) st = e->Dnorm.alloc((size_t)ns * ns);
  if (st == cudaSuccess) st = e->Dmax.alloc(2);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_direct scratch");
  launch_shell_norms(e, dD, e->Dnorm.p, e->Dmax.p, s);
  launch_final_to_cart(e, dD, e->Dcart.p, s);
  cudaMemsetAsync(e->Jcart.p, 0, sizeof(double) * nc * nc, s);
  cudaMemsetAsync(e->Kcart.p, 0, sizeof(double) * nc * nc, s);
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(e->Dmax.p + 1);
  e->last_counter = counter;
  cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  if ((st = e->class_work.alloc(3 * NPAIRCLASS * NPAIRCLASS)) != cudaSuccess)
    return check_cuda(e, st, "jk_direct work counters");
  cudaMemsetAsync(e->class_work.p, 0, sizeof(unsigned long long) * 3 * NPAIRCLASS * NPAIRCLASS, s);
  e->class_work_valid = true;
  JKParams P{};
  P.pp = prim_view(e);
  P.sh = shell_view(e);
  P.Dnorm = e->Dnorm.p;
  P.nshell = ns;
  P.Dmax = e->Dmax.p;
  P.Dc = e->Dcart.p;
  P.nc = nc;
  P.Jc = e->Jcart.p;
  P.Kc = e->Kcart.p;
  P.dstride = (size_t)nc * nc;
  P.precision = precision;
  P.boys = e->boys.p;
  P.counter = counter;
  P.kchunk = 128;  // one ket per thread: small classes still spread over the SMs
  launch_classes(e, s, [&](int A, int B, cudaStream_t cs) {
    JKParams Q = P;
    Q.bra = view(e->pcls[A]);
    Q.ket = view(e->pcls[B]);
    Q.same_class = (A == B);
    Q.work = e->class_work.p + 3 * (A * NPAIRCLASS + B);
    launch_jk(e, A, B, Q, e->pcls[A].npair, e->pcls[B].npair, cs);
  });
  // J = 1/4 (J + J^T) mult, K = 1/2 * 1/4 (K + K^T) mult  (src/fockbuild.cpp:146-149, 161-162)
  launch_cart_to_final_sym(e, e->Jcart.p, 0.25 * mult, dJ, s);
  launch_cart_to_final_sym(e, e->Kcart.p, 0.125 * mult, dK, s);
  return check_cuda(e, cudaGetLastError(), "jk_direct launch");
}

// J and K of two densities (UHF alpha and beta) from one pass over the shell
// quartets: UnrestrictedFock::formJKdirect (src/fockbuild.cpp:266-362), which
// screens with the shell-block norms of Da + Db and digests both densities from
// each integral batch.  Each J, K is w.r.t. its own full density.
int direct_jk_uhf_device(jk_engine* e, const double* dDa, const double* dDb, double precision, double mult,
                         double* dJa, double* dJb, double* dKa, double* dKb, cudaStream_t s) {
  const int n = e->obs.n_final, nc = e->obs.n_cart, ns = e->obs.nshell;
  const size_t ncc = (size_t)nc * nc, nn = (size_t)n * n;
  DevBuf<double> Dsum, Dc2, Jc2, Kc2;
  cudaError_t st = Dsum.alloc(nn);
  if (st == cudaSuccess) st = Dc2.alloc(2 * ncc);
  if (st == cudaSuccess) st = Jc2.alloc(2 * ncc);
  if (st == cudaSuccess) st = Kc2.alloc(2 * ncc);
  if (st == cudaSuccess) st = e->Dnorm.alloc((size_t)ns * ns);
  if (st == cudaSuccess) st = e->Dmax.alloc(2);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_direct_uhf scratch");
  launch_add(dDa, dDb, Dsum.p, nn, s);
  launch_shell_norms(e, Dsum.p, e->Dnorm.p, e->Dmax.p, s);
  launch_final_to_cart(e, dDa, Dc2.p, s);
  launch_final_to_cart(e, dDb, Dc2.p + ncc, s);
  cudaMemsetAsync(Jc2.p, 0, sizeof(double) * 2 * ncc, s);
  cudaMemsetAsync(Kc2.p, 0, sizeof(double) * 2 * ncc, s);
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(e->Dmax.p + 1);
  e->last_counter = counter;
  cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  JKParams P{};
  P.pp = prim_view(e);
  P.sh = shell_view(e);
  P.Dnorm = e->Dnorm.p;
  P.nshell = ns;
  P.Dmax = e->Dmax.p;
  P.Dc = Dc2.p;
  P.nc = nc;
  P.Jc = Jc2.p;
  P.Kc = Kc2.p;
  P.dstride = ncc;
  P.precision = precision;
  P.boys = e->boys.p;
  P.counter = counter;
  if ((st = e->class_work.alloc(3 * NPAIRCLASS * NPAIRCLASS)) != cudaSuccess)
    return check_cuda(e, st, "jk_direct_uhf work counters");
  cudaMemsetAsync(e->class_work.p, 0, sizeof(unsigned long long) * 3 * NPAIRCLASS * NPAIRCLASS, s);
  e->class_work_valid = true;
  launch_classes(e, s, [&](int A, int B, cudaStream_t cs) {
    JKParams Q = P;
    Q.bra = view(e->pcls[A]);
    Q.ket = view(e->pcls[B]);
    Q.same_class = (A == B);
    Q.work = e->class_work.p + 3 * (A * NPAIRCLASS + B);
    launch_jk(e, A, B, Q, e->pcls[A].npair, e->pcls[B].npair, cs, 2);
  });
  launch_cart_to_final_sym(e, Jc2.p, 0.25 * mult, dJa, s);
  launch_cart_to_final_sym(e, Jc2.p + ncc, 0.25 * mult, dJb, s);
  launch_cart_to_final_sym(e, Kc2.p, 0.125 * mult, dKa, s);
  launch_cart_to_final_sym(e, Kc2.p + ncc, 0.125 * mult, dKb, s);
  st = cudaGetLastError();
  if (st == cudaSuccess) st = cudaStreamSynchronize(s);  // the scratch dies on return
  return check_cuda(e, st, "jk_direct_uhf");
}

// ---------------------------------------------------------------- no-allocation variant
// Scratch of jk_direct_noalloc: one fixed array in device global memory.  Every
// GPU that loads this library holds it (6.8 MB) until the process exits, and
// every call on a device shares it.  Layout (in doubles): Cartesian D, J, K
// (NOALLOC_MAX_CART^2 each), the shell-block norms (NOALLOC_MAX_SHELLS^2), then
// Dmax and the quartet counter.
constexpr int NOALLOC_MAX_CART = 512;
constexpr int NOALLOC_MAX_SHELLS = 256;
constexpr size_t NOALLOC_CC = (size_t)NOALLOC_MAX_CART * NOALLOC_MAX_CART;
constexpr size_t NOALLOC_SS = (size_t)NOALLOC_MAX_SHELLS * NOALLOC_MAX_SHELLS;
constexpr size_t NOALLOC_DOUBLES = 3 * NOALLOC_CC + NOALLOC_SS + 2;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_DOUBLES];

// Device address of the scratch array on `device`, looked up once per device
// with that device current (the host-side symbol is not a device address).
static cudaError_t noalloc_scratch(int device, double** out) {
  static std::mutex mu;
  static std::vector<double*> addr;
  std::lock_guard<std::mutex> lock(mu);
  if ((int)addr.size() <= device) addr.resize(device + 1, nullptr);
  if (!addr[device]) {
    int prev = -1;
    cudaError_t st = cudaGetDevice(&prev);
    if (st == cudaSuccess && prev != device) st = cudaSetDevice(device);
    double* p = nullptr;
    if (st == cudaSuccess) st = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (prev >= 0 && prev != device) cudaSetDevice(prev);
    if (st != cudaSuccess) return st;
    addr[device] = p;
  }
  *out = addr[device];
  return cudaSuccess;
}

int direct_jk_noalloc(jk_engine* e, const double* dD, double precision, double mult, double* dJ, double* dK,
                      cudaStream_t s) {
  const int nc = e->obs.n_cart, ns = e->obs.nshell;
  if (nc > NOALLOC_MAX_CART || ns > NOALLOC_MAX_SHELLS)
    return set_error(e, JK_ERR_ARG,
                     "jk_direct_noalloc: basis too large for the fixed scratch (" + std::to_string(nc) +
                         " Cartesian functions, max " + std::to_string(NOALLOC_MAX_CART) + "; " + std::to_string(ns) +
                         " shells, max " + std::to_string(NOALLOC_MAX_SHELLS) + "); use jk_direct_device");
  // the array's address is per device: launching on another GPU than the
  // engine's would hand its kernels a foreign address
  int cur = -1;
  cudaError_t st = cudaGetDevice(&cur);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_direct_noalloc: cudaGetDevice");
  if (cur != e->device)
    return set_error(e, JK_ERR_ARG,
                     "jk_direct_noalloc: the current CUDA device (" + std::to_string(cur) +
                         ") is not the engine's device (" + std::to_string(e->device) + ")");
  double* base = nullptr;
  st = noalloc_scratch(e->device, &base);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_direct_noalloc: cudaGetSymbolAddress");
  double* Dc = base;
  double* Jc = base + NOALLOC_CC;
  double* Kc = base + 2 * NOALLOC_CC;
  double* Dn = base + 3 * NOALLOC_CC;
  double* Dmax = Dn + NOALLOC_SS;
  unsigned long long* counter = reinterpret_cast<unsigned long long*>(Dmax + 1);
  e->last_counter = counter;
  e->class_work_valid = false;  // this build keeps no per-class counters
  // the array keeps the previous call's contents: clear the accumulators
  launch_shell_norms(e, dD, Dn, Dmax, s);  // zeroes Dmax itself
  launch_final_to_cart(e, dD, Dc, s);
  cudaMemsetAsync(Jc, 0, sizeof(double) * nc * nc, s);
  cudaMemsetAsync(Kc, 0, sizeof(double) * nc * nc, s);
  cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
  JKParams P{};
  P.pp = prim_view(e);
  P.sh = shell_view(e);
  P.Dnorm = Dn;
  P.nshell = ns;
  P.Dmax = Dmax;
  P.Dc = Dc;
  P.nc = nc;
  P.Jc = Jc;
  P.Kc = Kc;
  P.precision = precision;
  P.boys = e->boys.p;
  P.counter = counter;
  P.dstride = NOALLOC_CC;
  P.kchunk = 128;  // one ket per thread: small classes still spread over the SMs
  launch_classes(e, s, [&](int A, int B, cudaStream_t cs) {
    JKParams Q = P;
    Q.bra = view(e->pcls[A]);
    Q.ket = view(e->pcls[B]);
    Q.same_class = (A == B);
    launch_jk(e, A, B, Q, e->pcls[A].npair, e->pcls[B].npair, cs);
  });
  launch_cart_to_final_sym(e, Jc, 0.25 * mult, dJ, s);
  launch_cart_to_final_sym(e, Kc, 0.125 * mult, dK, s);
  return check_cuda(e, cudaGetLastError(), "jk_direct_noalloc launch");
}

}  // namespace m2

using namespace m2;

extern "C" {

int jk_direct_uhf_device(jk_engine* e, const double* dDa, const double* dDb, double precision, double multiplier,
                         double* dJa, double* dJb, double* dKa, double* dKb, void* stream) {
  if (!e || !dDa || !dDb || !dJa || !dJb || !dKa || !dKb) return JK_ERR_ARG;
  if (!(precision >= 0.0)) return set_error(e, JK_ERR_ARG, "jk_direct_uhf: precision must be >= 0");
  PartitionScope part(e);
  return direct_jk_uhf_device(e, dDa, dDb, precision, multiplier, dJa, dJb, dKa, dKb,
                              stream ? (cudaStream_t)stream : e->stream);
}

int jk_direct_uhf(jk_engine* e, const double* Da, const double* Db, double precision, double multiplier, double* Ja,
                  double* Jb, double* Ka, double* Kb) {
  if (!e || !Da || !Db || !Ja || !Jb || !Ka || !Kb) return JK_ERR_ARG;
  const int n = e->obs.n_final;
  const size_t nn = (size_t)n * n, bytes = sizeof(double) * nn;
  DevBuf<double> d;
  cudaError_t st = d.alloc(6 * nn);
  if (st == cudaSuccess) st = cudaMemcpyAsync(d.p, Da, bytes, cudaMemcpyHostToDevice, e->stream);
  if (st == cudaSuccess) st = cudaMemcpyAsync(d.p + nn, Db, bytes, cudaMemcpyHostToDevice, e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_direct_uhf upload");
  int rc = jk_direct_uhf_device(e, d.p, d.p + nn, precision, multiplier, d.p + 2 * nn, d.p + 3 * nn, d.p + 4 * nn,
                                d.p + 5 * nn, nullptr);
  if (rc) return rc;
  double* outs[4] = {Ja, Jb, Ka, Kb};
  for (int k = 0; k < 4 && st == cudaSuccess; ++k)
    st = cudaMemcpyAsync(outs[k], d.p + (2 + k) * nn, bytes, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  return check_cuda(e, st, "jk_direct_uhf download");
}

int jk_last_class_work(const jk_engine* e, long long* out, int nmax, int* nwritten) {
  if (!e || !out || !nwritten) return JK_ERR_ARG;
  *nwritten = 0;
  if (!e->class_work_valid || !e->class_work.p) return JK_ERR_STATE;
  std::vector<unsigned long long> h(3 * NPAIRCLASS * NPAIRCLASS);
  if (cudaMemcpyAsync(h.data(), e->class_work.p, h.size() * sizeof(h[0]), cudaMemcpyDeviceToHost, e->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(e->stream) != cudaSuccess)
    return JK_ERR_CUDA;
  const int k = std::min<int>(nmax, (int)h.size());
  for (int i = 0; i < k; ++i) out[i] = (long long)h[i];
  *nwritten = k;
  return JK_OK;
}

int jk_direct_noalloc(jk_engine* e, const double* dD, double precision, double multiplier, double* dJ, double* dK,
                      void* stream) {
  if (!e || !dD || !dJ || !dK) return JK_ERR_ARG;
  if (!(precision >= 0.0)) return set_error(e, JK_ERR_ARG, "jk_direct_noalloc: precision must be >= 0");
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  PartitionScope part(e);
  return direct_jk_noalloc(e, dD, precision, multiplier, dJ, dK, s);
}

int jk_direct_device(jk_engine* e, const double* dD, double precision, double multiplier, double* dJ, double* dK,
                     void* stream) {
  if (!e || !dD || !dJ || !dK) return JK_ERR_ARG;
  if (!(precision >= 0.0)) return set_error(e, JK_ERR_ARG, "jk_direct: precision must be >= 0");
  cudaStream_t s = stream ? (cudaStream_t)stream : e->stream;
  PartitionScope part(e);
  return direct_jk_device(e, dD, precision, multiplier, dJ, dK, s);
}

int jk_direct_set_partition(jk_engine* e, int rank, int nranks) {
  if (!e) return JK_ERR_ARG;
  if (nranks < 1 || rank < 0 || rank >= nranks)
    return set_error(e, JK_ERR_ARG, "jk_direct_set_partition: need 0 <= rank < nranks");
  e->part_rank = rank;
  e->part_size = nranks;
  return JK_OK;
}

int jk_direct(jk_engine* e, const double* D, double precision, double multiplier, double* J, double* K) {
  if (!e || !D || !J || !K) return JK_ERR_ARG;
  const int n = e->obs.n_final;
  const size_t bytes = sizeof(double) * n * n;
  cudaError_t st = cudaSuccess;
  if (st == cudaSuccess) st = e->Dfinal.alloc((size_t)n * n);
  if (st == cudaSuccess) st = e->Jfinal.alloc((size_t)n * n);
  if (st == cudaSuccess) st = e->Kfinal.alloc((size_t)n * n);
  if (st == cudaSuccess) st = cudaMemcpyAsync(e->Dfinal.p, D, bytes, cudaMemcpyHostToDevice, e->stream);
  if (st != cudaSuccess) return check_cuda(e, st, "jk_direct upload");
  int rc = jk_direct_device(e, e->Dfinal.p, precision, multiplier, e->Jfinal.p, e->Kfinal.p, nullptr);
  if (rc) return rc;
  st = cudaMemcpyAsync(J, e->Jfinal.p, bytes, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaMemcpyAsync(K, e->Kfinal.p, bytes, cudaMemcpyDeviceToHost, e->stream);
  if (st == cudaSuccess) st = cudaStreamSynchronize(e->stream);
  return check_cuda(e, st, "jk_direct download");
}

}  // extern "C"
