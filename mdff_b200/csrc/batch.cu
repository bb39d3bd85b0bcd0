// batch.cu -- host side and C ABI of the batched engine (batch.cuh).
//
// Set-up runs the single engine's host set-up (setup.h) per configuration,
// then concatenates the per-ion and per-k tables.  One evaluation is a CUDA
// graph of three nodes: zero the work queue, zero the scalar slots, launch the
// persistent cluster kernel.  The launch shape (cluster size x threads per
// CTA) is chosen by an autotuner that times every candidate on the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/mdff_gpu.h"
#include "adjoint.cuh"
#include "batch.cuh"
#include "setup.h"

using namespace mdff;

namespace {

struct Shape {
  int cluster, threads;
};
const Shape kShapes[] = {{1, 256}, {2, 256}, {4, 256}, {8, 256},
                         {1, 512}, {2, 512}, {4, 512}, {8, 512}};

}  // namespace

struct mdff_batch {
  int device = 0, nconf = 0, ntot = 0, nmax = 0, mixed = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
  // host copies
  std::vector<BConf> conf;
  std::vector<int> order;
  std::vector<mdff_params> pconf;   // processed parameters per configuration
  std::vector<double> omega, coul_unit, press_unit;
  std::vector<int> lsr, lpolar, pset_of;
  // device
  BConf* d_conf = nullptr;
  int *d_order = nullptr, *d_queue = nullptr, *d_typ = nullptr, *d_ipol = nullptr;
  double *d_pos = nullptr, *d_q = nullptr, *d_pol = nullptr, *d_inv = nullptr;
  double4* d_dip = nullptr;
  NBPair* d_nb = nullptr;
  ESPair* d_es = nullptr;
  int4* d_rows = nullptr;
  double *d_Ak = nullptr;
  double4* d_kvec = nullptr;
  double4 *d_s = nullptr, *d_Estat = nullptr, *d_x = nullptr, *d_r = nullptr, *d_z = nullptr,
          *d_p = nullptr, *d_mu = nullptr, *d_E = nullptr;
  double2* d_tab64 = nullptr;
  float2* d_tab32 = nullptr;
  double2* d_rho = nullptr;
  double *d_force = nullptr, *d_part = nullptr, *d_out = nullptr, *d_pack = nullptr;
  double* h_out = nullptr;
  // launch
  Shape shape{2, 256};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  const double* graph_pos = nullptr;
  double* graph_force = nullptr;
  double ms_last = 0.0;
  bool have_pos = false;
  // fitting: parameter sets as given, fit parameters and their values
  std::vector<mdff_params> base;
  std::vector<double> cells;
  int nparam = 0;
  FitParam prm[kFitMax];
  std::vector<double> theta;
  double4 *d_w = nullptr, *d_rhs = nullptr, *d_lam = nullptr;
  double2 *d_ch = nullptr;  // 5 structure-factor channels of sum nk
  double *d_grad = nullptr, *d_info = nullptr, *d_gin = nullptr;
  long long ktot = 0;
  double ms_adjoint = 0.0;
};

namespace {

thread_local std::string g_berr;

#define BCK(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);         \
      return MDFF_ERR_CUDA;                                                \
    }                                                                      \
  } while (0)

template <typename T>
int balloc(mdff_batch* h, T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    h->err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
    return MDFF_ERR_NOMEM;
  }
  cudaMemsetAsync(*p, 0, n * sizeof(T), h->st);
  return MDFF_OK;
}
#define BALLOC(ptr, n)                   \
  do {                                   \
    int s_ = balloc(h, &(ptr), (n));     \
    if (s_) return s_;                   \
  } while (0)

template <typename T>
int bupload(mdff_batch* h, T** p, const std::vector<T>& v) {
  int s = balloc(h, p, v.size());
  if (s) return s;
  if (!v.empty()) BCK(cudaMemcpyAsync(*p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, h->st));
  return MDFF_OK;
}
#define BUPLOAD(ptr, vec)                \
  do {                                   \
    int s_ = bupload(h, &(ptr), (vec));  \
    if (s_) return s_;                   \
  } while (0)

__global__ void k_bpack3(const double4* __restrict__ v, int n, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[3 * i] = v[i].x;
  out[3 * i + 1] = v[i].y;
  out[3 * i + 2] = v[i].z;
}

BatchArgs make_args(mdff_batch* h, const double* d_pos, double* d_force) {
  BatchArgs a;
  a.nconf = h->nconf;
  a.ntot = h->ntot;
  a.conf = h->d_conf;
  a.order = h->d_order;
  a.queue = h->d_queue;
  a.pos = d_pos;
  a.typ = h->d_typ;
  a.q = h->d_q;
  a.ipol = h->d_ipol;
  a.pol = h->d_pol;
  a.inv = h->d_inv;
  a.dip = h->d_dip;
  a.nbtab = h->d_nb;
  a.estab = h->d_es;
  a.rows = h->d_rows;
  a.Ak = h->d_Ak;
  a.kvec = h->d_kvec;
  a.s = h->d_s;
  a.tab64 = h->d_tab64;
  a.tab32 = h->d_tab32;
  a.rho = h->d_rho;
  a.Estat = h->d_Estat;
  a.x = h->d_x;
  a.r = h->d_r;
  a.z = h->d_z;
  a.p = h->d_p;
  a.mu = h->d_mu;
  a.E = h->d_E;
  a.force = d_force;
  a.part = h->d_part;
  a.out = h->d_out;
  return a;
}

// persistent grid: as many clusters as fit on the device at once (at most one
// per configuration).  Attribute and occupancy queries happen here, outside
// any stream capture.
int prepare_shape(mdff_batch* h, Shape sh, int* nclusters) {
  size_t smem = batch_smem_bytes(h->nmax);
  void (*fn)(BatchArgs, int) = h->mixed ? k_batch<true> : k_batch<false>;
  BCK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = sh.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3(sh.threads);
  cfg.dynamicSmemBytes = smem;
  cfg.gridDim = dim3(sh.cluster);
  int ncl = 0;
  BCK(cudaOccupancyMaxActiveClusters(&ncl, (void*)fn, &cfg));
  if (ncl <= 0) {
    h->err = "launch shape does not fit on the device";
    return MDFF_ERR_CUDA;
  }
  *nclusters = std::min(ncl, h->nconf);
  return MDFF_OK;
}

int launch_batch(mdff_batch* h, const BatchArgs& a, Shape sh, int ncl, cudaStream_t st) {
  void (*fn)(BatchArgs, int) = h->mixed ? k_batch<true> : k_batch<false>;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = sh.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3(sh.threads);
  cfg.dynamicSmemBytes = batch_smem_bytes(h->nmax);
  cfg.stream = st;
  cfg.gridDim = dim3(sh.cluster * ncl);
  BCK(cudaLaunchKernelEx(&cfg, fn, a, h->nmax));
  return MDFF_OK;
}

// the evaluation as stream work: zero the queue and the slots, launch
int enqueue(mdff_batch* h, const double* d_pos, double* d_force, Shape sh, int ncl, cudaStream_t st) {
  BCK(cudaMemsetAsync(h->d_queue, 0, sizeof(int), st));
  BCK(cudaMemsetAsync(h->d_out, 0, sizeof(double) * kBSlots * h->nconf, st));
  return launch_batch(h, make_args(h, d_pos, d_force), sh, ncl, st);
}

int build_graph(mdff_batch* h, const double* d_pos, double* d_force) {
  if (h->exec) {
    cudaGraphExecDestroy(h->exec);
    h->exec = nullptr;
  }
  if (h->graph) {
    cudaGraphDestroy(h->graph);
    h->graph = nullptr;
  }
  int ncl = 0;
  int s = prepare_shape(h, h->shape, &ncl);
  if (s) return s;
  BCK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  s = enqueue(h, d_pos, d_force, h->shape, ncl, h->st);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(h->st, &g);
  if (s) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess) {
    h->err = std::string("graph capture: ") + cudaGetErrorString(e);
    return MDFF_ERR_CUDA;
  }
  h->graph = g;
  BCK(cudaGraphInstantiate(&h->exec, h->graph, 0));
  h->graph_pos = d_pos;
  h->graph_force = d_force;
  return MDFF_OK;
}

int run(mdff_batch* h, const double* d_pos, double* d_force) {
  int s;
  if (!h->exec || h->graph_pos != d_pos || h->graph_force != d_force)
    if ((s = build_graph(h, d_pos, d_force))) return s;
  BCK(cudaEventRecord(h->ev0, h->st));
  BCK(cudaGraphLaunch(h->exec, h->st));
  BCK(cudaEventRecord(h->ev1, h->st));
  BCK(cudaMemcpyAsync(h->h_out, h->d_out, sizeof(double) * kBSlots * h->nconf,
                      cudaMemcpyDeviceToHost, h->st));
  BCK(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->ms_last = ms;
  h->have_pos = true;
  return MDFF_OK;
}

// slots -> per-configuration outputs; status of the batch
int finish(mdff_batch* h, mdff_batch_conf* conf) {
  int status = MDFF_OK;
  for (int c = 0; c < h->nconf; ++c) {
    const double* sc = h->h_out + (size_t)c * kBSlots;
    int cata = sc[BS_CATA] != 0.0;
    int conv = (h->conf[c].flags & BF_POLAR) ? (sc[BS_CONV] != 0.0) : 1;
    if ((h->conf[c].flags & BF_WFC) && sc[BS_STAT] != 0.0) {
      status = (int)sc[BS_STAT];
      h->err = "configuration " + std::to_string(c) +
               ": a Wannier centre is missing for an ion of a type with lwfc > 0 "
               "(moment_from_pola.f90:731-737)";
    } else if (cata && status != MDFF_ERR_BAD_ARGS) {
      status = MDFF_ERR_CATASTROPHE;
    }
    else if (!conv && h->pconf[c].fail_on_nonconvergence && status == MDFF_OK)
      status = MDFF_ERR_NOT_CONVERGED;
    if (!conf) continue;
    mdff_result r;
    memset(&r, 0, sizeof(r));
    scalars_to_result(sc, h->pconf[c], h->lsr[c], h->lpolar[c], h->omega[c], h->coul_unit[c],
                      h->press_unit[c], &r);
    mdff_batch_conf& o = conf[c];
    o.u_lj = r.u_lj;
    o.vir_lj = r.vir_lj;
    o.u_bmhft = r.u_bmhft;
    o.vir_bmhft = r.vir_bmhft;
    o.u_coul = r.u_coul;
    o.u_pol = r.u_pol;
    o.pvirial_coul = r.pvirial_coul;
    memcpy(o.tau_nonb, r.tau_nonb, sizeof(r.tau_nonb));
    memcpy(o.tau_coul, r.tau_coul, sizeof(r.tau_coul));
    memcpy(o.tau, r.tau, sizeof(r.tau));
    o.rmsd = sc[BS_RMSD];
    o.n_pol_iter = (int)sc[BS_ITER];
    o.converged = conv;
    o.catastrophe = cata;
    o.nk = h->conf[c].nk;
    o.alphaES = h->pconf[c].alphaES;
    o.cutlongrange = h->pconf[c].cutlongrange;
    for (int d = 0; d < 3; ++d) o.kES[d] = h->pconf[c].kES[d];
    o.pad = 0;
  }
  if (status == MDFF_ERR_CATASTROPHE) h->err = "polarisation catastrophe (moment_from_pola.f90:176-216)";
  if (status == MDFF_ERR_BAD_ARGS) return status;
  if (status == MDFF_ERR_NOT_CONVERGED) h->err = "dipole solve did not converge";
  return status;
}

int create_impl(mdff_batch* h, const mdff_params* psets, int npsets, const mdff_batch_desc* d) {
  if (!psets || npsets <= 0 || !d || d->nconf <= 0 || !d->pset || !d->natmi || !d->cell_A) {
    h->err = "bad batch description";
    return MDFF_ERR_BAD_ARGS;
  }
  h->nconf = d->nconf;
  h->base.assign(psets, psets + npsets);
  h->cells.assign(d->cell_A, d->cell_A + 9 * (size_t)d->nconf);
  h->mixed = psets[0].precision == MDFF_PREC_MIXED ? 1 : 0;
  h->device = psets[0].device;
  int ndev = 0;
  // host set-up of every configuration first (validation needs no device)
  std::vector<int> typ, ipol;
  std::vector<double> q, pol, inv, Ak;
  std::vector<double4> dip, kvec;
  std::vector<NBPair> nb;
  std::vector<ESPair> es;
  std::vector<int4> rows;
  std::vector<double> cost(h->nconf);
  long long tab_total = 0;
  long long ktot = 0;
  int ntot = 0;
  h->conf.resize(h->nconf);
  h->pconf.resize(h->nconf);
  h->omega.resize(h->nconf);
  h->coul_unit.resize(h->nconf);
  h->press_unit.resize(h->nconf);
  h->lsr.resize(h->nconf);
  h->lpolar.resize(h->nconf);
  for (int c = 0; c < h->nconf; ++c) {
    int ps = d->pset[c];
    if (ps < 0 || ps >= npsets) {
      h->err = "pset index out of range";
      return MDFF_ERR_BAD_ARGS;
    }
    mdff_params p = psets[ps];
    // every parameter set's dipoles come from PCG: with kO_v1, kO_v2 or
    // kO_v4_1 selected the batch returns that algorithm's converged dipoles
    // (the same fixed point to the tolerance), not its iteration path, which
    // mdff_gpu_create reproduces (kO_v3 / kO_v4_2 stay rejected there)
    if (p.algo_moment_from_pola == MDFF_ALGO_KO_V1 || p.algo_moment_from_pola == MDFF_ALGO_KO_V2 ||
        p.algo_moment_from_pola == MDFF_ALGO_KO_V4_1)
      p.algo_moment_from_pola = MDFF_ALGO_SCF;
    h->pset_of.push_back(ps);
    long n = 0;
    for (int t = 0; t < MDFF_NTYPEMAX; ++t) {
      p.natmi[t] = (t < p.ntype) ? d->natmi[(size_t)c * MDFF_NTYPEMAX + t] : 0;
      n += p.natmi[t];
    }
    p.natm = (int)n;
    p.calc = MDFF_CALC_OTHER;
    if (p.ntype > MDFF_BATCH_MAXTYPES || n > MDFF_BATCH_MAXATM || n <= 0) {
      h->err = "configuration " + std::to_string(c) + ": ntype <= " +
               std::to_string(MDFF_BATCH_MAXTYPES) + " and 1 <= natm <= " +
               std::to_string(MDFF_BATCH_MAXATM) + " required";
      return MDFF_ERR_BAD_ARGS;
    }
    Setup S;
    const char* serr = nullptr;
    int s = setup_system(&p, d->cell_A + 9 * (size_t)c, S, &serr);
    if (s) {
      h->err = "configuration " + std::to_string(c) + ": " + serr;
      return s;
    }
    const mdff_params& P = S.p;
    h->pconf[c] = P;
    h->omega[c] = S.L.omega;
    h->coul_unit[c] = S.coul_unit;
    h->press_unit[c] = S.press_unit;
    h->lsr[c] = S.lsr;
    h->lpolar[c] = S.lpolar;
    BConf& B = h->conf[c];
    memset(&B, 0, sizeof(B));
    B.off = ntot;
    B.n = (int)n;
    B.ntype = P.ntype;
    int fl = 0;
    if (P.lcoulomb) fl |= BF_COUL;
    if (S.lsr) fl |= BF_SR;
    if (P.lbmhft || P.lbmhftd) fl |= BF_BMH;
    if (P.lbmhftd) fl |= BF_BMHFTD;
    if (P.lnmlj) fl |= BF_LJ;
    if (S.lpolar) fl |= BF_POLAR;
    if (S.task_qq) fl |= BF_QQ;
    if (S.task_qd) fl |= BF_QD;
    if (S.task_dd) fl |= BF_DD;
    if (P.lsurf) fl |= BF_SURF;
    if (P.thole_type != MDFF_THOLE_NONE) fl |= BF_THOLE;
    if (S.ldip_static) fl |= BF_DIPST;
    // Wannier centres (moment_from_pola.f90:130-147): a type with lwfc > 0
    for (int t = 0; t < P.ntype; ++t) {
      B.lwfc[t] = P.lwfc[t];
      if (P.lcoulomb && P.lwfc[t] > 0) fl |= BF_WFC;
    }
    B.ldip_wfc = P.ldip_wfc;
    B.rcut_wfc = P.rcut_wfc;
    B.flags = fl;
    B.trunc = P.trunc;
    B.maxit = P.cg_max_iter > 0 ? P.cg_max_iter : 200;
    B.tol = P.cg_tol > 0 ? P.cg_tol : P.conv_tol_ind;
    B.npol = S.npol;
    memcpy(B.A, S.L.A, sizeof(B.A));
    memcpy(B.B, S.L.B, sizeof(B.B));
    B.omega = S.L.omega;
    B.alpha = P.alphaES;
    B.rc2 = P.cutlongrange * P.cutlongrange;
    B.coul_unit = S.coul_unit;
    B.nb_off = (int)nb.size();
    B.es_off = (int)es.size();
    nb.insert(nb.end(), S.nb.begin(), S.nb.end());
    es.insert(es.end(), S.es.begin(), S.es.end());
    typ.insert(typ.end(), S.itype.begin(), S.itype.end());
    ipol.insert(ipol.end(), S.ipol.begin(), S.ipol.end());
    q.insert(q.end(), S.q.begin(), S.q.end());
    pol.insert(pol.end(), S.pol.begin(), S.pol.end());
    inv.insert(inv.end(), S.inv.begin(), S.inv.end());
    dip.insert(dip.end(), S.dip.begin(), S.dip.end());
    if (P.lcoulomb) {
      KMesh M;
      kmesh_of(P.kES, S.L.B, P.alphaES, M);
      if (P.kES[2] > 12 || P.kES[0] > 64 || P.kES[1] > 64) {
        h->err = "configuration " + std::to_string(c) + ": kES(3) <= 12 and kES(1:2) <= 64 required";
        return MDFF_ERR_BAD_ARGS;
      }
      B.nk = M.nk;
      B.nrows = (int)M.rows.size();
      B.row_off = (int)rows.size();
      B.k_off = (int)ktot;
      B.kx = P.kES[0];
      B.ky = P.kES[1];
      B.kz = P.kES[2];
      B.ntab = P.kES[0] + 1 + P.kES[1] + 1 + std::max(P.kES[2], 4) + 1;
      B.tab_off = tab_total;
      B.tab_ld = (int)n;
      tab_total += (long long)B.ntab * n;
      rows.insert(rows.end(), M.rows.begin(), M.rows.end());
      if (M.nk > 0) {
        Ak.insert(Ak.end(), M.Ak.begin(), M.Ak.begin() + M.nk);
        kvec.insert(kvec.end(), M.kv.begin(), M.kv.begin() + M.nk);
      }
      ktot += M.nk;
    }
    // cost model for the queue order: pair loops ~ n^2, k sums ~ n nk
    cost[c] = (double)n * n + 2.0 * (double)n * B.nk;
    ntot += (int)n;
    h->nmax = std::max(h->nmax, (int)n);
  }
  h->ntot = ntot;
  h->ktot = ktot;
  h->order.resize(h->nconf);
  std::iota(h->order.begin(), h->order.end(), 0);
  std::stable_sort(h->order.begin(), h->order.end(),
                   [&](int x, int y) { return cost[x] > cost[y]; });
  // device
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= h->device) {
    h->err = "no CUDA device";
    return MDFF_ERR_NO_DEVICE;
  }
  BCK(cudaSetDevice(h->device));
  BCK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
  BCK(cudaEventCreate(&h->ev0));
  BCK(cudaEventCreate(&h->ev1));
  BUPLOAD(h->d_conf, h->conf);
  BUPLOAD(h->d_order, h->order);
  BUPLOAD(h->d_typ, typ);
  BUPLOAD(h->d_ipol, ipol);
  BUPLOAD(h->d_q, q);
  BUPLOAD(h->d_pol, pol);
  BUPLOAD(h->d_inv, inv);
  BUPLOAD(h->d_dip, dip);
  BUPLOAD(h->d_nb, nb);
  BUPLOAD(h->d_es, es);
  BUPLOAD(h->d_rows, rows);
  BUPLOAD(h->d_Ak, Ak);
  BUPLOAD(h->d_kvec, kvec);
  BALLOC(h->d_queue, 1);
  BALLOC(h->d_pos, 3 * (size_t)ntot);
  BALLOC(h->d_s, ntot);
  BALLOC(h->d_Estat, ntot);
  BALLOC(h->d_x, ntot);
  BALLOC(h->d_r, ntot);
  BALLOC(h->d_z, ntot);
  BALLOC(h->d_p, ntot);
  BALLOC(h->d_mu, ntot);
  BALLOC(h->d_E, ntot);
  BALLOC(h->d_tab64, (size_t)std::max<long long>(tab_total, 1));
  if (h->mixed) BALLOC(h->d_tab32, (size_t)std::max<long long>(tab_total, 1));
  BALLOC(h->d_rho, (size_t)std::max<long long>(ktot, 1));
  BALLOC(h->d_force, 3 * (size_t)ntot);
  BALLOC(h->d_pack, 3 * (size_t)ntot);
  BALLOC(h->d_part, (size_t)h->nconf * kBMaxC * 2 * kBPart);
  BALLOC(h->d_out, (size_t)h->nconf * kBSlots);
  BCK(cudaMallocHost((void**)&h->h_out, sizeof(double) * kBSlots * h->nconf));
  if (batch_smem_bytes(h->nmax) > 227 * 1024) {
    h->err = "configurations too large for the shared-memory layout";
    return MDFF_ERR_BAD_ARGS;
  }
  BCK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

// the parameter set of configuration c with the fit parameters' values
mdff_params fitted_pset(const mdff_batch* h, int ps) {
  mdff_params p = h->base[ps];
  for (int k = 0; k < h->nparam; ++k) {
    const FitParam& f = h->prm[k];
    double v = h->theta[k];
    int a = f.t1, b = f.t2;
    switch (f.kind) {
      case FIT_A: p.Abmhftd[a][b] = p.Abmhftd[b][a] = v; break;
      case FIT_RHO: p.Bbmhftd[a][b] = p.Bbmhftd[b][a] = 1.0 / v; break;
      case FIT_C: p.Cbmhftd[a][b] = p.Cbmhftd[b][a] = v; break;
      case FIT_POL:
        for (int x = 0; x < 3; ++x)
          for (int y = 0; y < 3; ++y) p.poldip[a][x][y] = (x == y) ? v : 0.0;
        break;
      // field on dipole type a from charges of type b: tables (a,a,b) and (a,b,a)
      case FIT_TTB: p.pol_damp_b[a][a][b] = p.pol_damp_b[a][b][a] = v; break;
      case FIT_TTC: p.pol_damp_c[a][a][b] = p.pol_damp_c[a][b][a] = v; break;
      case FIT_QSCALE:
        for (int t = 0; t < MDFF_NTYPEMAX; ++t) p.qch[t] = h->base[ps].qch[t] * v;
        break;
    }
  }
  return p;
}

// rebuild the value tables of every configuration for the current theta
int refit_tables(mdff_batch* h) {
  std::vector<double> q, pol, inv;
  std::vector<NBPair> nb;
  std::vector<ESPair> es;
  for (int c = 0; c < h->nconf; ++c) {
    mdff_params p = fitted_pset(h, h->pset_of[c]);
    for (int t = 0; t < MDFF_NTYPEMAX; ++t) p.natmi[t] = h->pconf[c].natmi[t];
    p.natm = h->pconf[c].natm;
    p.calc = MDFF_CALC_OTHER;
    Setup S;
    const char* serr = nullptr;
    int s = setup_system(&p, h->cells.data() + 9 * (size_t)c, S, &serr);
    if (s) {
      h->err = "configuration " + std::to_string(c) + ": " + serr;
      return s;
    }
    h->pconf[c] = S.p;
    nb.insert(nb.end(), S.nb.begin(), S.nb.end());
    es.insert(es.end(), S.es.begin(), S.es.end());
    q.insert(q.end(), S.q.begin(), S.q.end());
    pol.insert(pol.end(), S.pol.begin(), S.pol.end());
    inv.insert(inv.end(), S.inv.begin(), S.inv.end());
  }
  BCK(cudaMemcpyAsync(h->d_nb, nb.data(), sizeof(NBPair) * nb.size(), cudaMemcpyHostToDevice, h->st));
  BCK(cudaMemcpyAsync(h->d_es, es.data(), sizeof(ESPair) * es.size(), cudaMemcpyHostToDevice, h->st));
  BCK(cudaMemcpyAsync(h->d_q, q.data(), sizeof(double) * q.size(), cudaMemcpyHostToDevice, h->st));
  BCK(cudaMemcpyAsync(h->d_pol, pol.data(), sizeof(double) * pol.size(), cudaMemcpyHostToDevice, h->st));
  BCK(cudaMemcpyAsync(h->d_inv, inv.data(), sizeof(double) * inv.size(), cudaMemcpyHostToDevice, h->st));
  BCK(cudaStreamSynchronize(h->st));
  return MDFF_OK;
}

void destroy_impl(mdff_batch* h) {
  if (!h) return;
  if (h->device >= 0) cudaSetDevice(h->device);
  if (h->st) cudaStreamSynchronize(h->st);
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  void* bufs[] = {h->d_conf, h->d_order, h->d_queue, h->d_typ, h->d_ipol, h->d_pos, h->d_q,
                  h->d_pol, h->d_inv, h->d_dip, h->d_nb, h->d_es, h->d_rows, h->d_Ak, h->d_kvec,
                  h->d_s, h->d_Estat, h->d_x, h->d_r, h->d_z, h->d_p, h->d_mu, h->d_E,
                  h->d_tab64, h->d_tab32, h->d_rho, h->d_force, h->d_part, h->d_out, h->d_pack,
                  h->d_w, h->d_rhs, h->d_lam, h->d_ch, h->d_grad, h->d_info, h->d_gin};
  for (void* b : bufs)
    if (b) cudaFree(b);
  if (h->h_out) cudaFreeHost(h->h_out);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

}  // namespace

extern "C" {

int mdff_gpu_batch_create(const mdff_params* psets, int npsets, const mdff_batch_desc* desc,
                          mdff_batch_handle* out) {
  if (!out) return MDFF_ERR_BAD_ARGS;
  *out = nullptr;
  mdff_batch* h = new mdff_batch();
  int s = create_impl(h, psets, npsets, desc);
  if (s) {
    g_berr = h->err;
    destroy_impl(h);
    return s;
  }
  *out = h;
  return MDFF_OK;
}

int mdff_gpu_batch_engforce_device(mdff_batch_handle h, const double* d_pos, double* d_force,
                                   double* d_mu, double* d_ef, mdff_batch_conf* conf) {
  if (!h || !d_pos || !d_force) return MDFF_ERR_BAD_ARGS;
  BCK(cudaSetDevice(h->device));
  int s = run(h, d_pos, d_force);
  if (s) return s;
  int nb = (h->ntot + 255) / 256;
  if (d_mu) {
    k_bpack3<<<nb, 256, 0, h->st>>>(h->d_mu, h->ntot, d_mu);
    BCK(cudaGetLastError());
  }
  if (d_ef) {
    k_bpack3<<<nb, 256, 0, h->st>>>(h->d_E, h->ntot, d_ef);
    BCK(cudaGetLastError());
  }
  BCK(cudaStreamSynchronize(h->st));
  return finish(h, conf);
}

int mdff_gpu_batch_engforce(mdff_batch_handle h, const double* rx, const double* ry,
                            const double* rz, double* fx, double* fy, double* fz, double* mu,
                            double* ef, mdff_batch_conf* conf) {
  if (!h || !rx || !ry || !rz || !fx || !fy || !fz) return MDFF_ERR_BAD_ARGS;
  BCK(cudaSetDevice(h->device));
  size_t nb = sizeof(double) * h->ntot;
  BCK(cudaMemcpyAsync(h->d_pos, rx, nb, cudaMemcpyHostToDevice, h->st));
  BCK(cudaMemcpyAsync(h->d_pos + h->ntot, ry, nb, cudaMemcpyHostToDevice, h->st));
  BCK(cudaMemcpyAsync(h->d_pos + 2 * (size_t)h->ntot, rz, nb, cudaMemcpyHostToDevice, h->st));
  int s = run(h, h->d_pos, h->d_force);
  if (s) return s;
  BCK(cudaMemcpyAsync(fx, h->d_force, nb, cudaMemcpyDeviceToHost, h->st));
  BCK(cudaMemcpyAsync(fy, h->d_force + h->ntot, nb, cudaMemcpyDeviceToHost, h->st));
  BCK(cudaMemcpyAsync(fz, h->d_force + 2 * (size_t)h->ntot, nb, cudaMemcpyDeviceToHost, h->st));
  int nblk = (h->ntot + 255) / 256;
  if (mu) {
    k_bpack3<<<nblk, 256, 0, h->st>>>(h->d_mu, h->ntot, h->d_pack);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(mu, h->d_pack, 3 * nb, cudaMemcpyDeviceToHost, h->st));
  }
  if (ef) {
    k_bpack3<<<nblk, 256, 0, h->st>>>(h->d_E, h->ntot, h->d_pack);
    BCK(cudaGetLastError());
    BCK(cudaMemcpyAsync(ef, h->d_pack, 3 * nb, cudaMemcpyDeviceToHost, h->st));
  }
  BCK(cudaStreamSynchronize(h->st));
  return finish(h, conf);
}

int mdff_gpu_batch_tune(mdff_batch_handle h, int* cluster, int* threads, double* ms) {
  if (!h) return MDFF_ERR_BAD_ARGS;
  if (!h->have_pos) {
    h->err = "tune needs one evaluation first (its positions are reused)";
    return MDFF_ERR_BAD_ARGS;
  }
  BCK(cudaSetDevice(h->device));
  const double* pos = h->graph_pos;
  double* force = h->graph_force;
  double best = 1e300;
  Shape bs = h->shape;
  for (const Shape& sh : kShapes) {
    // warm-up, then the median of three
    int ncl = 0;
    int s = prepare_shape(h, sh, &ncl);
    if (s == MDFF_OK) s = enqueue(h, pos, force, sh, ncl, h->st);
    if (s) {
      h->err.clear();
      cudaGetLastError();
      continue;
    }
    float t[3];
    for (int r = 0; r < 3; ++r) {
      BCK(cudaEventRecord(h->ev0, h->st));
      if ((s = enqueue(h, pos, force, sh, ncl, h->st))) return s;
      BCK(cudaEventRecord(h->ev1, h->st));
      BCK(cudaEventSynchronize(h->ev1));
      cudaEventElapsedTime(&t[r], h->ev0, h->ev1);
    }
    std::sort(t, t + 3);
    if (t[1] < best) {
      best = t[1];
      bs = sh;
    }
  }
  h->shape = bs;
  int s = build_graph(h, pos, force);
  if (s) return s;
  if (cluster) *cluster = bs.cluster;
  if (threads) *threads = bs.threads;
  if (ms) *ms = best;
  return MDFF_OK;
}

int mdff_gpu_batch_set_shape(mdff_batch_handle h, int cluster, int threads) {
  if (!h) return MDFF_ERR_BAD_ARGS;
  bool ok = false;
  for (const Shape& sh : kShapes) ok = ok || (sh.cluster == cluster && sh.threads == threads);
  if (!ok) {
    h->err = "shape must be cluster 1/2/4/8 x threads 256/512";
    return MDFF_ERR_BAD_ARGS;
  }
  h->shape = Shape{cluster, threads};
  if (h->exec) {
    cudaGraphExecDestroy(h->exec);
    h->exec = nullptr;
  }
  return MDFF_OK;
}

int mdff_gpu_batch_info(mdff_batch_handle h, int* ntot, int* nconf, int* cluster, int* threads,
                        double* ms_last) {
  if (!h) return MDFF_ERR_BAD_ARGS;
  if (ntot) *ntot = h->ntot;
  if (nconf) *nconf = h->nconf;
  if (cluster) *cluster = h->shape.cluster;
  if (threads) *threads = h->shape.threads;
  if (ms_last) *ms_last = h->ms_last;
  return MDFF_OK;
}

int mdff_gpu_batch_fit_define(mdff_batch_handle h, int nparam, const int* kind, const int* t1,
                              const int* t2) {
  if (!h || nparam < 0 || nparam > kFitMax || (nparam > 0 && (!kind || !t1 || !t2))) {
    if (h) h->err = "0 <= nparam <= 16 and kind/t1/t2 arrays required";
    return MDFF_ERR_BAD_ARGS;
  }
  for (int c = 0; c < h->nconf; ++c) {
    if (h->pconf[c].lsurf) {
      h->err = "the fit gradient does not cover the surface term (lsurf)";
      return MDFF_ERR_BAD_ARGS;
    }
    if (h->pconf[c].thole_type != MDFF_THOLE_NONE) {
      h->err = "the fit gradient does not cover Thole functions";
      return MDFF_ERR_UNSUPPORTED;
    }
    if (h->conf[c].flags & BF_WFC) {
      h->err = "the fit gradient does not cover Wannier centres";
      return MDFF_ERR_UNSUPPORTED;
    }
  }
  int ntmin = MDFF_NTYPEMAX;
  for (const auto& p : h->base) ntmin = std::min(ntmin, p.ntype);
  h->nparam = nparam;
  h->theta.assign(nparam, 0.0);
  // initial values from the parameter set of the first configuration
  const mdff_params& p0 = h->base[h->pset_of[0]];
  for (int k = 0; k < nparam; ++k) {
    FitParam f{kind[k], t1[k], t2[k], 0};
    bool types_ok = f.t1 >= 0 && f.t1 < ntmin && f.t2 >= 0 && f.t2 < ntmin;
    if (f.kind < FIT_A || f.kind > FIT_QSCALE || (f.kind != FIT_QSCALE && !types_ok)) {
      h->err = "fit parameter " + std::to_string(k) + ": unknown kind or type index";
      h->nparam = 0;
      return MDFF_ERR_BAD_ARGS;
    }
    h->prm[k] = f;
    int a = f.t1, b = f.t2;
    switch (f.kind) {
      case FIT_A: h->theta[k] = p0.Abmhftd[a][b]; break;
      case FIT_RHO: h->theta[k] = p0.Bbmhftd[a][b] != 0.0 ? 1.0 / p0.Bbmhftd[a][b] : 0.0; break;
      case FIT_C: h->theta[k] = p0.Cbmhftd[a][b]; break;
      case FIT_POL: h->theta[k] = p0.poldip[a][0][0]; break;
      case FIT_TTB: h->theta[k] = p0.pol_damp_b[a][b][a]; break;
      case FIT_TTC: h->theta[k] = p0.pol_damp_c[a][b][a]; break;
      case FIT_QSCALE: h->theta[k] = 1.0; break;
    }
  }
  BCK(cudaSetDevice(h->device));
  if (!h->d_w) {
    size_t nk = (size_t)std::max<long long>(h->ktot, 1);
    BALLOC(h->d_w, h->ntot);
    BALLOC(h->d_rhs, h->ntot);
    BALLOC(h->d_lam, h->ntot);
    BALLOC(h->d_ch, 5 * nk);
    BALLOC(h->d_grad, (size_t)h->nconf * kFitMax);
    BALLOC(h->d_info, (size_t)h->nconf * 4);
    BALLOC(h->d_gin, (size_t)h->nconf + 6 * (size_t)h->ntot);
  }
  return MDFF_OK;
}

int mdff_gpu_batch_fit_set(mdff_batch_handle h, const double* theta) {
  if (!h || !theta) return MDFF_ERR_BAD_ARGS;
  for (int k = 0; k < h->nparam; ++k) {
    if (!std::isfinite(theta[k]) || (h->prm[k].kind == FIT_RHO && theta[k] <= 0.0) ||
        (h->prm[k].kind == FIT_POL && theta[k] <= 0.0)) {
      h->err = "fit parameter " + std::to_string(k) + " out of its domain";
      return MDFF_ERR_BAD_ARGS;
    }
  }
  h->theta.assign(theta, theta + h->nparam);
  BCK(cudaSetDevice(h->device));
  return refit_tables(h);
}

int mdff_gpu_batch_fit_get(mdff_batch_handle h, double* theta) {
  if (!h || !theta) return MDFF_ERR_BAD_ARGS;
  for (int k = 0; k < h->nparam; ++k) theta[k] = h->theta[k];
  return MDFF_OK;
}

int mdff_gpu_batch_adjoint(mdff_batch_handle h, const double* gE, const double* gF,
                           const double* gmu, int on_device, double* grad, double* grad_conf) {
  if (!h || !gE || !gF || !grad) return MDFF_ERR_BAD_ARGS;
  if (!h->have_pos || h->nparam == 0) {
    h->err = "adjoint needs fit_define and a forward evaluation first";
    return MDFF_ERR_BAD_ARGS;
  }
  BCK(cudaSetDevice(h->device));
  const double *dgE = gE, *dgF = gF, *dgmu = gmu;
  if (!on_device) {
    double* g0 = h->d_gin;
    BCK(cudaMemcpyAsync(g0, gE, sizeof(double) * h->nconf, cudaMemcpyHostToDevice, h->st));
    BCK(cudaMemcpyAsync(g0 + h->nconf, gF, sizeof(double) * 3 * h->ntot, cudaMemcpyHostToDevice, h->st));
    dgE = g0;
    dgF = g0 + h->nconf;
    if (gmu) {
      BCK(cudaMemcpyAsync(g0 + h->nconf + 3 * (size_t)h->ntot, gmu, sizeof(double) * 3 * h->ntot,
                          cudaMemcpyHostToDevice, h->st));
      dgmu = g0 + h->nconf + 3 * (size_t)h->ntot;
    }
  }
  AdjArgs J;
  J.gE = dgE;
  J.gF = dgF;
  J.gmu = dgmu;
  J.w = h->d_w;
  J.rhs = h->d_rhs;
  J.lam = h->d_lam;
  size_t nk = (size_t)std::max<long long>(h->ktot, 1);
  J.rq = h->d_ch;
  J.rm = h->d_ch + nk;
  J.sq = h->d_ch + 2 * nk;
  J.sm = h->d_ch + 3 * nk;
  J.rl = h->d_ch + 4 * nk;
  J.grad = h->d_grad;
  J.info = h->d_info;
  J.qscale = 1.0;
  for (int k = 0; k < h->nparam; ++k)
    if (h->prm[k].kind == FIT_QSCALE) J.qscale = h->theta[k];
  J.tol_rel = 1e-12;
  J.nparam = h->nparam;
  for (int k = 0; k < kFitMax; ++k) J.prm[k] = (k < h->nparam) ? h->prm[k] : FitParam{-1, 0, 0, 0};
  // launch: persistent clusters of the forward's block size; the cluster is
  // widened until the clusters of all configurations cover the SMs twice (a
  // fitting batch of tens of boxes would otherwise leave most SMs idle)
  Shape sh = h->shape;
  {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    while (sh.cluster < kBMaxC && (long)h->nconf * sh.cluster < 2L * nsm) sh.cluster *= 2;
  }
  size_t smem = batch_smem_extra_offset(h->nmax) + sizeof(double4) * h->nmax;
  if (smem > 227 * 1024) {
    h->err = "configurations too large for the adjoint's shared-memory layout";
    return MDFF_ERR_BAD_ARGS;
  }
  BCK(cudaFuncSetAttribute(k_batch_adjoint, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = sh.cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.blockDim = dim3(sh.threads);
  cfg.dynamicSmemBytes = smem;
  cfg.gridDim = dim3(sh.cluster);
  int ncl = 0;
  BCK(cudaOccupancyMaxActiveClusters(&ncl, (void*)k_batch_adjoint, &cfg));
  if (ncl <= 0) {
    h->err = "adjoint launch shape does not fit on the device";
    return MDFF_ERR_CUDA;
  }
  ncl = std::min(ncl, h->nconf);
  cfg.gridDim = dim3(sh.cluster * ncl);
  cfg.stream = h->st;
  BatchArgs a = make_args(h, h->graph_pos, h->graph_force);
  BCK(cudaMemsetAsync(h->d_queue, 0, sizeof(int), h->st));
  BCK(cudaEventRecord(h->ev0, h->st));
  BCK(cudaLaunchKernelEx(&cfg, k_batch_adjoint, a, J, h->nmax));
  BCK(cudaEventRecord(h->ev1, h->st));
  std::vector<double> gc((size_t)h->nconf * kFitMax);
  BCK(cudaMemcpyAsync(gc.data(), h->d_grad, sizeof(double) * gc.size(), cudaMemcpyDeviceToHost, h->st));
  BCK(cudaStreamSynchronize(h->st));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, h->ev0, h->ev1);
  h->ms_adjoint = ms;
  for (int k = 0; k < h->nparam; ++k) {
    double s = 0.0;
    for (int c = 0; c < h->nconf; ++c) s += gc[(size_t)c * kFitMax + k];
    grad[k] = s;
  }
  if (grad_conf)
    for (int c = 0; c < h->nconf; ++c)
      for (int k = 0; k < h->nparam; ++k) grad_conf[(size_t)c * h->nparam + k] = gc[(size_t)c * kFitMax + k];
  return MDFF_OK;
}

const char* mdff_gpu_batch_last_error(mdff_batch_handle h) {
  return h ? h->err.c_str() : g_berr.c_str();
}

void mdff_gpu_batch_destroy(mdff_batch_handle h) { destroy_impl(h); }

}  // extern "C"
