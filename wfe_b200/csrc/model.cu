// ModelT<R>: device buffers, the RK3 large step and its CUDA-graph replay,
// and the operator-level entry points of one case on one B200.
//
// Buffer roles.  Three full states rotate with period three: at the start of
// a step S[perm[0]] holds time n (N); stage 0 writes S[perm[1]], stage 1
// reads it and writes S[perm[2]], stage 2 reads that and writes S[perm[1]],
// which becomes the next N.  The reference instead copies time n into a work
// state at every stage (integrator.cpp:93-94: nine device copies per stage)
// and swaps pointers, which is why its CUDA-graph attempt was reverted; the
// fixed rotation lets three captured graphs (one per phase) replay any number
// of steps.  Inside a stage the acoustic loop reads time n from N on its first
// substep and double-buffers u, v (U2, V2) and rotates pi' through three
// buffers (X.pip, P1, P2), so the last substep lands in the stage output X
// without any copy.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>

#include "core.cuh"
#include "kernels.cuh"
#include "model.hpp"

namespace wfe {

// Kernel variants picked by the autotuner.  Every variant computes the same
// values with the same arithmetic; only launch shapes differ.
struct Tune {
  int tend_variant = 0;  // 0 fused tendencies, 1 momentum + scalar launches, 2 with TMA-staged
                         // scalars, 3 fused with two cells per thread
  int column_cx = 0;     // acoustic column tile shape index (launch_acoustic_column)
  int persist = 0;       // ensembles: 0 one block per work item, 1 persistent grid, 2 members' own
                         // graphs on concurrent streams, 3 members' own graphs one after another
  int uv_variant = 0;    // forward u, v: 0 thread per face pair in 16 x 16 x 1 blocks, 1 persistent
                         // pipelined tiles, 2 thread per face pair in 32 x 2 x 4 blocks
  bool done = false;
};


namespace {
std::mutex g_tune_mu;
std::map<std::string, Tune> g_tune_cache;

std::string tune_cache_path() {
  const char* p = std::getenv("WFE_TUNE_CACHE");
  if (p && *p) return p;
  const char* h = std::getenv("HOME");
  return std::string(h && *h ? h : "/tmp") + "/.wfe_b200_tune.txt";
}

bool tune_lookup(const std::string& key, Tune* t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune_cache.find(key);
  if (it != g_tune_cache.end()) {
    *t = it->second;
    return true;
  }
  std::ifstream f(tune_cache_path());
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    std::string k;
    Tune v;
    if (ss >> k >> v.tend_variant >> v.column_cx && k == key) {
      if (!(ss >> v.persist)) v.persist = 0;
      if (!(ss >> v.uv_variant)) v.uv_variant = 0;
      v.done = true;
      g_tune_cache[key] = v;
      *t = v;
      return true;
    }
  }
  return false;
}

void tune_store(const std::string& key, const Tune& t) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = t;
  // best effort: the cache file is an optimisation only (its directory must exist)
  std::ofstream f(tune_cache_path(), std::ios::app);
  if (f) f << key << " " << t.tend_variant << " " << t.column_cx << " " << t.persist << " "
           << t.uv_variant << "\n";
}
}  // namespace

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda
// link); null when the driver does not provide it
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static std::once_flag once;
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e__ = (call);                                                     \
    if (e__ != cudaSuccess) return fail(std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

template <typename R>
class ModelT final : public Model {
 public:
  ~ModelT() override { release(); }

  int init(const CaseSetup& cs, int device) {
    cs_ = &cs;
    g_ = cs.g;
    hp_ = cs.p;
    L_ = make_layout(g_.nx, g_.ny, g_.nz);
    if (L_.n3() >= kMaxIndexedPoints)
      return fail("grid too large: a padded field must hold fewer than 2^31 points");
    dev_ = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    if (prepare_acoustic_column<R>(g_.nz) || prepare_kessler<R>(g_.nz) || prepare_sfc<R>(g_.nz))
      return fail("nz too large for the column kernels' shared memory");
    tma_ok_ = tensor_map_encoder() && prepare_acoustic_column_tma<R>(g_.nz) == 0;
    fused_ok_ = prepare_acoustic_fused<R>(g_.nz) == 0;
    pipe_ok_ = tensor_map_encoder() && prepare_acoustic_pipe<R>(g_.nz) == 0;
    uvp_ok_ = tensor_map_encoder() && prepare_acoustic_uv_pipe<R>() == 0;
    tend_tma_ok_ = tensor_map_encoder() && tend_scal_tma_smem<R>() <= 227 * 1024 &&
                   prepare_tend_scal_tma<R>() == 0;
    CK(cudaMalloc(&tma_err_, sizeof(unsigned)));
    CK(cudaMemset(tma_err_, 0, sizeof(unsigned)));
    const size_t n3 = L_.n3(), n2 = L_.n2(), n1 = L_.pz;
    // metric
    R* mbuf = alloc(4 * n1 + 8 * n2);
    if (!mbuf) return 1;
    const std::vector<double>* m1[4] = {&cs.m.zeta_w, &cs.m.zeta_c, &cs.m.dzeta_c, &cs.m.dzeta_w};
    const std::vector<double>* m2[8] = {&cs.m.h, &cs.m.hx, &cs.m.hy, &cs.m.hx_u,
                                        &cs.m.hy_v, &cs.m.jac, &cs.m.fcor, &cs.m.mapf};
    R* mp[12];
    for (int q = 0; q < 4; ++q) {
      mp[q] = mbuf + q * n1;
      if (put1d(mp[q], *m1[q])) return 1;
    }
    for (int q = 0; q < 8; ++q) {
      mp[4 + q] = mbuf + 4 * n1 + q * n2;
      if (put2d(mp[4 + q], *m2[q])) return 1;
    }
    dm_ = DMetric<R>{mp[0], mp[1], mp[2], mp[3], mp[4], mp[5], mp[6], mp[7],
                     mp[8], mp[9], mp[10], mp[11], (R)cs.m.zt};
    // base state
    const std::vector<double>* b3[9] = {&cs.b.thb, &cs.b.pib, &cs.b.rhob, &cs.b.dthbdz, &cs.b.thbw,
                                        &cs.b.rhobw, &cs.b.thvb, &cs.b.thvbw, &cs.b.qvb};
    R* bp[10];
    for (int q = 0; q < 9; ++q) {
      bp[q] = alloc(n3);
      if (!bp[q] || put3d(bp[q], *b3[q])) return 1;
    }
    bp[9] = alloc(n1);
    if (!bp[9] || put1d(bp[9], cs.b.ub)) return 1;
    db_ = DBase<R>{bp[0], bp[1], bp[2], bp[3], bp[4], bp[5], bp[6], bp[7], bp[8], bp[9]};
    // parameters
    dp_.diff_K = (R)hp_.diff_K;
    dp_.rayleigh_zd = (R)hp_.rayleigh_zd;
    dp_.rayleigh_alpha = (R)hp_.rayleigh_alpha;
    dp_.acoustic_beta = (R)hp_.acoustic_beta;
    dp_.acoustic_smdiv = (R)hp_.acoustic_smdiv;
    dp_.cstar = (R)hp_.cstar;
    dp_.w_abort = (R)hp_.w_abort;
    dp_.acoustic_ns = hp_.acoustic_ns;
    dp_.coriolis_use_ub = hp_.coriolis_use_ub ? 1 : 0;
    dp_.bc_x_open = hp_.bc_x_open;
    dp_.bc_y_open = hp_.bc_y_open;
    dp_.moisture = hp_.moisture;
    dp_.microphysics = hp_.microphysics;
    dp_.pd_moist = hp_.pd_moist;
    dp_.w_damping = hp_.w_damping;
    // prognostic states, tendencies, scratch
    for (int s = 0; s < 3; ++s)
      for (int f = 0; f < 8; ++f)
        if (!(S_[s][f] = alloc(n3))) return 1;
    for (int f = 0; f < 8; ++f)
      if (!(T_[f] = alloc(n3))) return 1;
    for (R** p : {&mfx_, &mfy_, &mfz_, &U2_, &V2_, &P1_, &P2_, &TH2_})
      if (!(*p = alloc(n3))) return 1;
    if (hp_.pd_moist)
      for (int s = 0; s < 3; ++s)
        if (!(ratio_[s] = alloc(n3))) return 1;
    // run-constant acoustic coefficients (kernels.cu:915-927)
    for (R** p : {&rtjx_, &rtjy_, &kt3_, &aw_})
      if (!(*p = alloc(n3))) return 1;
    R* scratch = alloc(n3);
    if (!scratch) return 1;
    launch_acoustic_coef<R>(L_, db_, dm_, scratch, rtjx_, rtjy_, kt3_, aw_, st_);
    CK(cudaStreamSynchronize(st_));
    CK(cudaGetLastError());
    {
      // per-level reciprocals and terrain-following factors of the metric
      std::vector<double> lv[7];
      for (auto& v : lv) v.assign(n1, 0.0);
      const double zt = cs.m.zt;
      // Rayleigh sponge coefficient (src/dynamics/kernels.cu:42-48)
      auto sponge = [&](double zeta) {
        const double zd = hp_.rayleigh_zd;
        if (zd < 0 || zeta <= zd || zt <= zd) return 0.0;
        double sn = std::sin(1.5707963267948966 * (zeta - zd) / (zt - zd));
        return hp_.rayleigh_alpha * sn * sn;
      };
      for (size_t q = 0; q < n1; ++q) {
        const double dzc = cs.m.dzeta_c[q], dzw = cs.m.dzeta_w[q];
        lv[0][q] = dzc != 0 ? 1.0 / dzc : 0.0;
        lv[1][q] = dzw != 0 ? 1.0 / dzw : 0.0;
        lv[2][q] = 1.0 - cs.m.zeta_w[q] / zt;
        lv[3][q] = 1.0 - cs.m.zeta_c[q] / zt;
        if (q >= 1 && q + 1 < n1) {
          const double d2 = cs.m.zeta_c[q + 1] - cs.m.zeta_c[q - 1];
          lv[4][q] = d2 != 0 ? 1.0 / d2 : 0.0;
        }
        lv[5][q] = sponge(cs.m.zeta_c[q]);
        lv[6][q] = sponge(cs.m.zeta_w[q]);
      }
      R* lb = alloc(7 * n1);
      if (!lb) return 1;
      for (int q = 0; q < 7; ++q)
        if (put1d(lb + q * n1, lv[q])) return 1;
      co_ = DCoef<R>{rtjx_,      rtjy_,      kt3_,       aw_,        lb,
                     lb + n1,    lb + 2 * n1, lb + 3 * n1, lb + 4 * n1, lb + 5 * n1,
                     lb + 6 * n1, (R)(1.0 / g_.dx), (R)(1.0 / g_.dy)};
    }
    if (level_tables()) return 1;
    if (!(rain_ = alloc(n2))) return 1;
    CK(cudaMalloc(&clock_, CLK_N * sizeof(double)));
    CK(cudaMemset(clock_, 0, CLK_N * sizeof(double)));
    CK(cudaMalloc(&wd_, sizeof(unsigned int)));
    CK(cudaMalloc(&mass_planes_, (size_t)g_.nz * sizeof(double)));
    CK(cudaMalloc(&mass_, sizeof(double)));
    CK(cudaMallocHost(&stage_, n3 * sizeof(R)));
    // initial state
    for (int f = 0; f < 8; ++f)
      if (upload(ROLE_STATE, f, cs.state[f].data())) return 1;
    return 0;
  }

  const RefGrid& grid() const override { return g_; }
  bool fp64() const override { return sizeof(R) == 8; }
  size_t pitched_count() const override { return L_.n3(); }
  void pitched_dims(int* px, int* py, int* pz) const override {
    *px = L_.px;
    *py = L_.py;
    *pz = L_.pz;
  }
  long launches_per_step() const override { return launches_; }

  // ------------------------------------------------------------ transfers
  R* field_ptr(int role, int field) {
    if (field < 0 || field > 7) return nullptr;
    switch (role) {
      case ROLE_STATE: return S_[perm_[0]][field];
      case ROLE_TEND: return T_[field];
      case ROLE_WORK: return S_[perm_[1]][field];
      case ROLE_PIPREV: return piprev_ ? piprev_ : S_[perm_[0]][4];
      case ROLE_LIN: return lin_map_ ? static_cast<R*>(lin_map_(S_[perm_[0]][field])) : nullptr;
      default: return nullptr;
    }
  }

  int upload(int role, int field, const double* ref) override {
    R* d = field_ptr(role, field);
    if (!d) return fail("bad role/field");
    to_pitched(ref, stage_, true);
    CK(cudaMemcpyAsync(d, stage_, L_.n3() * sizeof(R), cudaMemcpyHostToDevice, st_));
    CK(cudaStreamSynchronize(st_));
    return 0;
  }

  int download(int role, int field, double* ref) override {
    R* d = field_ptr(role, field);
    if (!d) return fail("bad role/field");
    CK(cudaMemcpyAsync(stage_, d, L_.n3() * sizeof(R), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    from_pitched(stage_, ref);
    return 0;
  }

  int download_interior(int role, int field, void* host, bool f32) override {
    R* d = field_ptr(role, field);
    if (!d) return fail("bad role/field");
    const int nzl = field == 2 ? g_.nz + 1 : g_.nz;
    // only the interior planes cross PCIe
    const size_t off = L_.at(-kOX, -kOY, 0), cnt = (size_t)nzl * L_.plane();
    CK(cudaMemcpyAsync(stage_ + off, d + off, cnt * sizeof(R), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    const size_t row = (size_t)g_.nx;
    for (int k = 0; k < nzl; ++k)
      for (int j = 0; j < g_.ny; ++j) {
        const R* src = stage_ + L_.at(0, j, k);
        size_t o = ((size_t)k * g_.ny + j) * row;
        if (f32 == (sizeof(R) == 4)) {
          std::memcpy((char*)host + o * sizeof(R), src, row * sizeof(R));
        } else if (f32) {
          float* dst = (float*)host + o;
          for (size_t i = 0; i < row; ++i) dst[i] = (float)src[i];
        } else {
          double* dst = (double*)host + o;
          for (size_t i = 0; i < row; ++i) dst[i] = (double)src[i];
        }
      }
    return 0;
  }

  int upload_interior(int role, int field, const void* host, bool f32) override {
    R* d = field_ptr(role, field);
    if (!d) return fail("bad role/field");
    const int nzl = field == 2 ? g_.nz + 1 : g_.nz;
    // the block crosses the host link as one copy into a device staging
    // buffer; a kernel scatters it into the interior points (ghosts and
    // padding keep their values).  Synchronous: the caller may reuse `host`.
    const size_t bytes = (size_t)nzl * g_.ny * g_.nx * (f32 ? 4 : 8);
    if (up_cap_ < bytes) {
      if (up_buf_) cudaFree(up_buf_);
      up_buf_ = nullptr;
      up_cap_ = 0;
      CK(cudaMalloc(&up_buf_, bytes));
      up_cap_ = bytes;
    }
    CK(cudaMemcpyAsync(up_buf_, host, bytes, cudaMemcpyHostToDevice, st_));
    launch_unpack_interior<R>(up_buf_, L_, nzl, d, f32, st_);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st_));
    return 0;
  }

  int snapshot_begin(int n, const int* fields, void* const* host, bool f32) override {
    if (snapshot_wait()) return 1;
    if (!cs_st_) CK(cudaStreamCreateWithFlags(&cs_st_, cudaStreamNonBlocking));
    if (!snap_ev_) CK(cudaEventCreateWithFlags(&snap_ev_, cudaEventDisableTiming));
    const size_t es = f32 ? 4 : 8;
    std::vector<size_t> off(n), bytes(n);
    size_t total = 0;
    for (int q = 0; q < n; ++q) {
      const int f = fields[q];
      size_t cnt;
      if (f >= 0 && f < 8) cnt = (size_t)(f == 2 ? g_.nz + 1 : g_.nz) * g_.ny * g_.nx;
      else if (f >= 100 && field2d(f - 100)) cnt = (size_t)g_.ny * g_.nx;
      else return fail("snapshot: bad field " + std::to_string(f));
      off[q] = total;
      bytes[q] = cnt * es;
      total += (bytes[q] + 255) / 256 * 256;
    }
    if (total > snap_cap_) {
      if (snap_buf_) cudaFree(snap_buf_);
      snap_buf_ = nullptr;
      snap_cap_ = 0;
      CK(cudaMalloc(&snap_buf_, total));
      snap_cap_ = total;
    }
    for (int q = 0; q < n; ++q) {
      const int f = fields[q];
      char* dst = static_cast<char*>(snap_buf_) + off[q];
      if (f < 8) launch_pack_interior<R>(S_[perm_[0]][f], L_, f == 2 ? g_.nz + 1 : g_.nz, dst, f32, st_);
      else launch_pack_interior2d<R>(field2d(f - 100), L_, dst, f32, st_);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(snap_ev_, st_));
    CK(cudaStreamWaitEvent(cs_st_, snap_ev_, 0));
    for (int q = 0; q < n; ++q)
      CK(cudaMemcpyAsync(host[q], static_cast<char*>(snap_buf_) + off[q], bytes[q],
                         cudaMemcpyDeviceToHost, cs_st_));
    return 0;
  }

  int snapshot_wait() override {
    if (cs_st_) CK(cudaStreamSynchronize(cs_st_));
    return 0;
  }

  int upload_state_raw(int field, const void* host) override {
    if (field < 0 || field > 7) return fail("bad field");
    CK(cudaMemcpyAsync(S_[perm_[0]][field], host, L_.n3() * sizeof(R), cudaMemcpyHostToDevice, st_));
    return 0;
  }
  int download_state_raw(int field, void* host) override {
    if (field < 0 || field > 7) return fail("bad field");
    CK(cudaMemcpyAsync(host, S_[perm_[0]][field], L_.n3() * sizeof(R), cudaMemcpyDeviceToHost, st_));
    return 0;
  }

  R* field2d(int which) {
    switch (which) {
      case F2_RAIN: return rain_;
      case F2_TSK: return sf_.tsk;
      case F2_PBLH: return sf_.pblh;
      case F2_T2M: return sf_.t2m;
      case F2_U10: return sf_.u10;
      case F2_WGT: return wgt_;
      default: return nullptr;
    }
  }

  int download2d(int which, double* ref2) override {
    R* d = field2d(which);
    if (!d) return fail("2D field not available");
    std::vector<R> h(L_.n2());
    CK(cudaMemcpyAsync(h.data(), d, L_.n2() * sizeof(R), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    for (int j = -3; j < g_.ny + 3; ++j)
      for (int i = -3; i < g_.nx + 3; ++i) ref2[g_.idx2(i, j)] = (double)h[L_.at2(i, j)];
    return 0;
  }

  int upload2d(int which, const double* ref2) override {
    R* d = field2d(which);
    if (!d) return fail("2D field not available");
    return put2d(d, std::vector<double>(ref2, ref2 + g_.n2()));
  }

  // ------------------------------------------------------------- stepping
  int step(double dt, double t) override {
    if (autotune(dt)) return 1;
    launch_clock(clock_, t, t_lo_, t_hi_, dt, 0, st_);
    launches_ = 1;
    if (enqueue_step((R)dt)) return 1;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st_));
    return check_tma();
  }

  int run(int nsteps, double dt, double t0) override {
    if (autotune(dt)) return 1;
    launch_clock(clock_, t0, t_lo_, t_hi_, dt, 0, st_);
    return graph_steps(nsteps, dt);
  }

  // nsteps graph-replayed steps on the member's stream, the clock running on
  // from its last value (the ensemble's concurrent mode; run() sets it first)
  int graph_steps(int nsteps, double dt) {
    if (!graphs_valid_ || graph_dt_ != dt) {
      for (auto& ge : gexec_)
        if (ge) {
          cudaGraphExecDestroy(ge);
          ge = nullptr;
        }
      graphs_valid_ = true;
      graph_dt_ = dt;
    }
    for (int s = 0; s < nsteps; ++s) {
      int ph = phase_;
      if (!gexec_[ph]) {
        int saved[3] = {perm_[0], perm_[1], perm_[2]};
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        launches_ = 0;
        int rc = enqueue_step((R)dt);
        launch_clock(clock_, 0, 0, 0, 0, 1, st_);
        ++launches_;
        cudaError_t ce = cudaStreamEndCapture(st_, &gr);
        if (rc) return 1;
        if (ce != cudaSuccess) return fail(std::string("graph capture: ") + cudaGetErrorString(ce));
        CK(cudaGraphInstantiate(&gexec_[ph], gr, 0));
        cudaGraphDestroy(gr);
        glaunches_ = launches_;
        // enqueue_step advanced the rotation during capture; restore it
        perm_[0] = saved[0];
        perm_[1] = saved[1];
        perm_[2] = saved[2];
        phase_ = ph;
      }
      CK(cudaGraphLaunch(gexec_[ph], st_));
      advance_rotation();
    }
    launches_ = glaunches_;
    CK(cudaGetLastError());
    return 0;
  }

  int time_run(int nsteps, double dt, double t0, double* ms) override {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st_));
    int rc = run(nsteps, dt, t0);
    CK(cudaEventRecord(e1, st_));
    CK(cudaEventSynchronize(e1));
    float f = 0;
    CK(cudaEventElapsedTime(&f, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = f;
    return rc;
  }

  // One step captured into a CUDA graph with an event-record node before and
  // after every kernel, replayed once: the per-kernel times of a replayed
  // step (the timed runs replay graphs too), not of direct launches.
  int kernel_times(double dt, double t, std::vector<std::string>* names, std::vector<double>* ms,
                   std::vector<int>* counts) override {
    if (autotune(dt)) return 1;
    launch_clock(clock_, t, t_lo_, t_hi_, dt, 0, st_);
    prof_.clear();
    profiling_ = true;
    const int ph = phase_;
    const int saved[3] = {perm_[0], perm_[1], perm_[2]};
    cudaGraph_t gr = nullptr;
    CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    launches_ = 1;
    int rc = enqueue_step((R)dt);
    cudaError_t ce = cudaStreamEndCapture(st_, &gr);
    profiling_ = false;
    if (rc) return rc;
    if (ce != cudaSuccess) return fail(std::string("graph capture: ") + cudaGetErrorString(ce));
    perm_[0] = saved[0];
    perm_[1] = saved[1];
    perm_[2] = saved[2];
    phase_ = ph;
    cudaGraphExec_t ge = nullptr;
    CK(cudaGraphInstantiate(&ge, gr, 0));
    cudaGraphDestroy(gr);
    CK(cudaGraphLaunch(ge, st_));
    advance_rotation();
    CK(cudaStreamSynchronize(st_));
    cudaGraphExecDestroy(ge);
    if (check_tma()) return 1;
    names->clear();
    ms->clear();
    counts->clear();
    for (auto& pr : prof_) {
      float f = 0;
      CK(cudaEventElapsedTime(&f, pr.e0, pr.e1));
      size_t q = 0;
      while (q < names->size() && (*names)[q] != pr.name) ++q;
      if (q == names->size()) {
        names->push_back(pr.name);
        ms->push_back(0);
        counts->push_back(0);
      }
      (*ms)[q] += f;
      (*counts)[q] += 1;
      cudaEventDestroy(pr.e0);
      cudaEventDestroy(pr.e1);
    }
    prof_.clear();
    return 0;
  }

  int sync() override {
    CK(cudaStreamSynchronize(st_));
    CK(cudaGetLastError());
    return check_tma();
  }

  // a TMA tile that did not arrive in time leaves the flag set
  int check_tma() {
    if (!tma_err_) return 0;
    unsigned e = 0;
    CK(cudaMemcpy(&e, tma_err_, sizeof(e), cudaMemcpyDeviceToHost));
    if (e) return fail("acoustic column: a TMA tile load timed out");
    return 0;
  }

  int absmax(int field, float* out) override {
    R* d = field_ptr(ROLE_STATE, field);
    if (!d) return fail("bad field");
    CK(cudaMemsetAsync(wd_, 0, sizeof(unsigned int), st_));
    launch_absmax<R>(d, L_.n3(), wd_, st_);
    unsigned int bits = 0;
    CK(cudaMemcpyAsync(&bits, wd_, sizeof(bits), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    std::memcpy(out, &bits, sizeof(float));
    return 0;
  }

  int absmax_begin(int field, int slot) override {
    if (slot < 0 || slot > 1) return fail("absmax slot must be 0 or 1");
    R* d = field_ptr(ROLE_STATE, field);
    if (!d) return fail("bad field");
    if (!wd_async_) {
      // per slot: the blocks' maximum and their count (left zero by every
      // launch); the result lands in mapped page-locked memory
      CK(cudaMalloc(&wd_async_, 4 * sizeof(unsigned int)));
      CK(cudaMemset(wd_async_, 0, 4 * sizeof(unsigned int)));
      CK(cudaHostAlloc(&wd_host_, 2 * sizeof(unsigned int), cudaHostAllocMapped));
      CK(cudaHostGetDevicePointer(reinterpret_cast<void**>(&wd_host_dev_), wd_host_, 0));
      for (auto& e : wd_ev_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    launch_absmax_to_host<R>(d, L_.n3(), wd_async_ + 2 * slot, wd_host_dev_ + slot, st_);
    CK(cudaGetLastError());
    CK(cudaEventRecord(wd_ev_[slot], st_));
    return 0;
  }

  int absmax_end(int slot, float* out) override {
    if (slot < 0 || slot > 1 || !wd_async_) return fail("absmax_end without absmax_begin");
    CK(cudaEventSynchronize(wd_ev_[slot]));
    unsigned int bits = *reinterpret_cast<volatile unsigned int*>(wd_host_ + slot);
    std::memcpy(out, &bits, sizeof(float));
    return 0;
  }

  int dry_mass(double* out) override {
    R** s = S_[perm_[0]];
    launch_dry_mass<R>(L_, db_, dm_, s[4], s[3], s[5], s[6], s[7], dp_.moisture, (R)g_.dx,
                       (R)g_.dy, mass_planes_, mass_, st_);
    CK(cudaMemcpyAsync(out, mass_, sizeof(double), cudaMemcpyDeviceToHost, st_));
    CK(cudaStreamSynchronize(st_));
    return 0;
  }

  // ------------------------------------------------------------ boundary
  int set_boundary(const double* const lo[5], const double* const hi[5], const double* wgt,
                   double t_lo, double t_hi) override {
    for (int v = 0; v < 5; ++v) {
      if (!lo_[v] && !(lo_[v] = alloc(L_.n3()))) return 1;
      if (!hi_[v] && !(hi_[v] = alloc(L_.n3()))) return 1;
      if (put3d(lo_[v], std::vector<double>(lo[v], lo[v] + g_.npts()))) return 1;
      if (put3d(hi_[v], std::vector<double>(hi[v], hi[v] + g_.npts()))) return 1;
    }
    if (!wgt_ && !(wgt_ = alloc(L_.n2()))) return 1;
    if (put2d(wgt_, std::vector<double>(wgt, wgt + g_.n2()))) return 1;
    t_lo_ = t_lo;
    t_hi_ = t_hi;
    bdy_on_ = true;
    graphs_valid_ = false;
    ++gen_;
    launch_clock(clock_, 0, t_lo, t_hi, 0, 0, st_);
    return sync();
  }

  int set_boundary_hi(const double* const hi[5], double t_lo, double t_hi) override {
    // BdyManager::update: the old upper targets become the lower ones
    // (src/dynamics/boundary.cpp:83-89); buffers swap, so graphs recapture
    if (!bdy_on_) return fail("boundary not set");
    for (int v = 0; v < 5; ++v) {
      std::swap(lo_[v], hi_[v]);
      if (put3d(hi_[v], std::vector<double>(hi[v], hi[v] + g_.npts()))) return 1;
    }
    t_lo_ = t_lo;
    t_hi_ = t_hi;
    graphs_valid_ = false;
    ++gen_;
    return 0;
  }

  int clear_boundary() override {
    if (!bdy_on_) return 0;
    bdy_on_ = false;
    graphs_valid_ = false;
    ++gen_;
    return 0;
  }

  // the scratch of the one-thread-per-column surface kernels, which a batched
  // launch runs when the ensemble's deepest column does not fit in shared
  // memory
  int ensure_sfc_scratch() {
    if (!sfc_on_ || sf_.scratch) return 0;
    return (sf_.scratch = alloc(sfc_scratch_count<R>(L_))) ? 0 : 1;
  }

  int enable_physics(const double* tsk, const double* land, const double* lat, const double* lon,
                     const double* soilw, double start_hour, int doy, bool nonlocal) override {
    // SfcPBL::init (src/physics/surface.cu:440-482); inputs interior ny*nx
    const size_t n2 = L_.n2();
    for (R** p : {&sf_.tsk, &sf_.tdeep, &sf_.land, &sf_.lat, &sf_.lon, &sf_.soilw, &sf_.cdv,
                  &sf_.pblh, &sf_.t2m, &sf_.u10})
      if (!*p && !(*p = alloc(n2))) return 1;
    if (!sf_.km && !(sf_.km = alloc(L_.n3()))) return 1;
    if (!sf_.soilt && !(sf_.soilt = alloc(4 * n2))) return 1;
    if (sfc_needs_scratch<R>(g_.nz) && !sf_.scratch && !(sf_.scratch = alloc(sfc_scratch_count<R>(L_))))
      return 1;
    auto pad = [&](const double* in) {
      std::vector<double> o(g_.n2(), 0.0);
      for (int j = 0; j < g_.ny; ++j)
        for (int i = 0; i < g_.nx; ++i) o[g_.idx2(i, j)] = in[(size_t)j * g_.nx + i];
      return o;
    };
    if (put2d(sf_.tsk, pad(tsk)) || put2d(sf_.tdeep, pad(tsk)) || put2d(sf_.land, pad(land)) ||
        put2d(sf_.lat, pad(lat)) || put2d(sf_.lon, pad(lon)) || put2d(sf_.soilw, pad(soilw)))
      return 1;
    for (int lyr = 0; lyr < 4; ++lyr)
      if (put2d(sf_.soilt + lyr * n2, pad(tsk))) return 1;
    sf_.start_hour = start_hour;
    sf_.doy = doy;
    sf_.nonlocal = nonlocal;
    sfc_on_ = true;
    graphs_valid_ = false;
    ++gen_;
    return sync();
  }

  // ----------------------------------------------------------- operators
  int op_apply_bcs() override {
    GhostJob<R> job = ghost_job(S_[perm_[0]], true);
    launch_fill_ghosts<R>(L_, job, dp_.bc_x_open, dp_.bc_y_open, st_);
    return sync();
  }

  int op_tendencies(double dt, double t) override {
    R** s = S_[perm_[0]];
    launch_clock(clock_, t, t_lo_, t_hi_, dt, 0, st_);
    tendencies(s, s, nullptr, (R)dt, (R)0, true);
    return sync();
  }

  int op_acoustic(double dtau, int nsub) override {
    R** N = S_[perm_[0]];
    R** X = S_[perm_[1]];
    if (acoustic(N, X, (R)dtau, nsub, true)) return 1;
    return sync();
  }

  int op_moisture_stage(double dt) override {
    R** N = S_[perm_[0]];
    R** X = S_[perm_[1]];
    for (int q = 5; q < 8; ++q) launch_axpy<R>(N[q], T_[q], (R)dt, X[q], L_.n3(), st_);
    return sync();
  }

  int op_kessler(double dt) override {
    if (kessler(S_[perm_[0]], (R)dt)) return 1;
    return sync();
  }

  int op_sfc(double dt, double t) override {
    if (!sfc_on_) return fail("surface physics not enabled");
    launch_clock(clock_, t - dt, t_lo_, t_hi_, dt, 0, st_);
    if (surface(S_[perm_[0]], (R)dt)) return 1;
    return sync();
  }

  // ----------------------------------------------------- batched ensembles
  // The launches of one step from the current rotation phase, recorded
  // instead of issued; the rotation is left unchanged.
  int record_step(double dt, std::vector<Rec>* out) override {
    const int saved[3] = {perm_[0], perm_[1], perm_[2]};
    const int ph = phase_;
    const long l = launches_;
    rec_ = out;
    int rc = enqueue_step((R)dt);
    rec_ = nullptr;
    launches_ = l;
    perm_[0] = saved[0];
    perm_[1] = saved[1];
    perm_[2] = saved[2];
    phase_ = ph;
    return rc;
  }
  void rotate() override { advance_rotation(); }
  int phase() const override { return phase_; }
  std::vector<std::pair<void*, size_t>> state_buffers() const override {
    std::vector<std::pair<void*, size_t>> v;
    const size_t n3 = L_.n3();
    for (int s = 0; s < 3; ++s)
      for (int f = 0; f < 8; ++f) v.push_back({S_[s][f], n3});
    for (int f = 0; f < 8; ++f) v.push_back({T_[f], n3});
    for (R* p : {mfx_, mfy_, mfz_, U2_, V2_, P1_, P2_}) v.push_back({p, n3});
    return v;
  }
  void* state_field(int field) override {
    return (field >= 0 && field < 8) ? S_[perm_[0]][field] : nullptr;
  }
  void* stream_handle() const override { return st_; }
  void variants(int out[4]) const override {
    out[0] = tune_.done ? tune_.tend_variant : -1;
    out[1] = tune_.done ? tune_.column_cx : -1;
    out[2] = tune_.done ? tune_.uv_variant : -1;
    out[3] = (lvl_tab_ != nullptr ? 1 : 0) | (db_.lvl != nullptr ? 2 : 0);
  }
  // chunked column variants follow the fused ones; -1 for other variants
  int chunked_index(int v) const {
    const int f = v - acoustic_column_shapes() - 1 - acoustic_fused_shapes();
    return (f >= 0 && f < acoustic_chunked_shapes()) ? f : -1;
  }
  bool chunked_usable(int v) const {
    const int f = chunked_index(v);
    return f >= 0 && acoustic_chunked_fits<R>(g_.nz, f);
  }
  // pipelined column variants follow the chunked ones; -1 for other variants
  int pipe_index(int v) const {
    const int f = v - acoustic_column_shapes() - 1 - acoustic_fused_shapes() - acoustic_chunked_shapes();
    return (f >= 0 && f < acoustic_pipe_shapes()) ? f : -1;
  }
  // parallel-solve column variants follow the pipelined ones; -1 otherwise
  int pcr_index(int v) const {
    const int f = v - acoustic_column_shapes() - 1 - acoustic_fused_shapes() - acoustic_chunked_shapes() -
                  acoustic_pipe_shapes();
    return (f >= 0 && f < acoustic_pcr_shapes()) ? f : -1;
  }
  bool pcr_usable(int v) const {
    const int f = pcr_index(v);
    return f >= 0 && acoustic_pcr_fits<R>(g_.nz, f);
  }
  // pipelined parallel-solve column variants follow those; -1 otherwise
  int pipe_pcr_index(int v) const {
    const int f = v - acoustic_column_shapes() - 1 - acoustic_fused_shapes() - acoustic_chunked_shapes() -
                  acoustic_pipe_shapes() - acoustic_pcr_shapes();
    return (f >= 0 && f < acoustic_pipe_pcr_shapes()) ? f : -1;
  }
  bool pipe_pcr_usable(int v) const {
    const int f = pipe_pcr_index(v);
    return pipe_ok_ && f >= 0 &&
           acoustic_pipe_pcr_smem<R>(f, g_.nz, dp_.moisture != 0, bdy_on_, lvl_tab_ != nullptr) > 0;
  }
  bool pipe_usable(int v) const {
    const int f = pipe_index(v);
    return pipe_ok_ && f >= 0 &&
           acoustic_pipe_smem<R>(f, g_.nz, dp_.moisture != 0, bdy_on_, lvl_tab_ != nullptr) > 0;
  }
  bool fused_usable(int v) const {
    const int f = v - acoustic_column_shapes() - 1;
    return fused_ok_ && f >= 0 && f < acoustic_fused_shapes() && acoustic_fused_fits<R>(g_.nz, f);
  }
  void set_lin_map(std::function<void*(const void*)> map) override { lin_map_ = std::move(map); }
  bool linearisable(std::string* why) const override {
    if (dp_.moisture && dp_.pd_moist) *why = "the positive-definite moisture limiter is not linearised";
    else if (bdy_on_) *why = "Davies relaxation is not linearised";
    else if (sfc_on_) *why = "the surface physics is not linearised";
    else if (dp_.w_damping) *why = "w damping is not linearised";
    else return true;
    return false;
  }
  long generation() const { return gen_; }
  double* clock_ptr() const { return clock_; }
  int tune_for(double dt) { return autotune(dt); }
  double bdy_t_lo() const { return t_lo_; }
  double bdy_t_hi() const { return t_hi_; }
  cudaStream_t stream() const { return st_; }
  int device() const { return dev_; }
  const Layout& layout() const { return L_; }
  // members whose signatures match record the same launch sequence
  std::string batch_signature() const {
    std::ostringstream k;
    k << "m" << dp_.moisture << "mp" << dp_.microphysics << "pd" << dp_.pd_moist << "b" << bdy_on_
      << "s" << sfc_on_ << "ns" << hp_.acoustic_ns;
    return k.str();
  }

 private:
  // ------------------------------------------------------------ autotuner
  // Times each kernel variant on the live buffers before the first step.  The
  // trial launches read time n and write only scratch, tendencies and the
  // stage-output state, which the step overwrites.  WFE_TUNE=0 keeps defaults.
  std::string tune_key() const {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, dev_);
    std::ostringstream k;
    std::string name = prop.name;
    for (char& ch : name)
      if (ch == ' ') ch = '_';
    k << "v8|" << name << "|" << g_.nx << "x" << g_.ny << "x" << g_.nz << "|" << (sizeof(R) * 8) << "|m"
      << dp_.moisture << "pd" << dp_.pd_moist << "b" << bdy_on_ << "d" << (dp_.diff_K > 0) << "x"
      << (pcr_allowed() ? 0 : 1);
    return k.str();
  }

  template <class F>
  int time_ms(F&& f, float* best) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    *best = 1e30f;
    // best of three timings of eight calls each: one call of a small grid's
    // variant takes a few microseconds, the size of the events' own jitter
    for (int rep = 0; rep < 3; ++rep) {
      CK(cudaEventRecord(e0, st_));
      for (int it = 0; it < 8; ++it)
        if (f()) return 1;
      // a variant whose launch is refused (its resources do not fit) is
      // never the fastest
      const bool refused = cudaGetLastError() != cudaSuccess;
      CK(cudaEventRecord(e1, st_));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (refused) {
        *best = 1e30f;
        break;
      }
      if (ms < *best) *best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return 0;
  }

  // whether the tuner may pick a column variant that is not bit-identical
  // to the others (the parallel-solve kernels): WFE_EXACT_COLUMN=0
  static bool pcr_allowed() {
    const char* e = std::getenv("WFE_EXACT_COLUMN");
    return e && e[0] == '0';
  }

  // WFE_COLUMN_VARIANT=<n> forces the acoustic variant (0..5 column tile
  // shapes, 6 the TMA-staged column, 7..9 the fused substep kernel in three
  // tile shapes, 10..12 the chunked column kernel, 13..15 the persistent
  // pipelined column kernel, 16..18 the parallel-solve column kernel and
  // 19..22 its pipelined form, both equal to the others up to rounding),
  // WFE_UV_VARIANT=<n> the forward u, v kernel (0
  // thread per face pair in 16 x 16 x 1 blocks, 1 persistent pipelined tiles,
  // 2 thread per face pair in 32 x 2 x 4 blocks) and WFE_TEND_VARIANT=<n>
  // the tendency variant (0 fused, 1 split, 2 momentum + TMA-staged scalars,
  // 3 fused with two cells per thread)
  // after tuning, for tests and experiments
  int autotune(double dt) {
    const bool first = !tune_.done;
    int rc = autotune_variants(dt);
    const char* cv = std::getenv("WFE_COLUMN_VARIANT");
    if (first && cv && *cv) {
      const int v = std::atoi(cv);
      if (v >= 0 && (v < acoustic_column_shapes() || (v == acoustic_column_shapes() && tma_ok_) ||
                     fused_usable(v) || chunked_usable(v) || pipe_usable(v) || pcr_usable(v) ||
                     pipe_pcr_usable(v)))
        tune_.column_cx = v;
    }
    const char* uvv = std::getenv("WFE_UV_VARIANT");
    if (first && uvv && *uvv) {
      const int v = std::atoi(uvv);
      if (v == 0 || (v == 1 && uvp_ok_) || v == 2) tune_.uv_variant = v;
    }
    const char* tv = std::getenv("WFE_TEND_VARIANT");
    if (first && tv && *tv) {
      const int v = std::atoi(tv);
      if (v >= 0 && (v < 2 || (v == 2 && tend_tma_usable()) || v == 3)) tune_.tend_variant = v;
    }
    return rc;
  }

  int autotune_variants(double dt) {
    if (tune_.done) return 0;
    tune_.done = true;
    const char* env = std::getenv("WFE_TUNE");
    if (env && env[0] == '0') return 0;
    const std::string key = tune_key();
    Tune cached;
    if (tune_lookup(key, &cached)) {
      tune_ = cached;
      return 0;
    }
    R** N = S_[perm_[0]];
    R** X = S_[perm_[1]];
    long saved = launches_;
    GhostJob<R> job = ghost_job(N, false);
    launch_fill_ghosts<R>(L_, job, dp_.bc_x_open, dp_.bc_y_open, st_);
    float best = 1e30f;
    // 0 fused, 1 split, 2 momentum + TMA-staged scalars, 3 fused with two
    // cells per thread
    for (int v = 0; v < 4; ++v) {
      if (v == 2 && !tend_tma_usable()) continue;
      float ms;
      tune_.tend_variant = v;
      if (time_ms([&] { tendencies(N, N, X, (R)dt, (R)dt / 3, false); return 0; }, &ms)) return 1;
      if (ms < best) {
        best = ms;
        cached.tend_variant = v;
      }
    }
    best = 1e30f;
    const int ns = hp_.acoustic_ns > 1 ? hp_.acoustic_ns : 1;
    // 0 and 2: one thread per face pair in square and slab-shaped blocks;
    // 1: the persistent pipelined tiles
    for (int v = 0; v < 3; ++v) {
      if (v == 1 && !uvp_ok_) continue;
      float ms;
      tune_.uv_variant = v;
      if (time_ms([&] { return acoustic(N, X, (R)dt / (R)ns, 1, false); }, &ms)) return 1;
      if (ms < best) {
        best = ms;
        cached.uv_variant = v;
      }
    }
    tune_.uv_variant = cached.uv_variant;
    best = 1e30f;
    // tile shapes, the TMA-staged column, the fused substep kernels
    const int nvar = acoustic_column_shapes() + 1 + acoustic_fused_shapes() + acoustic_chunked_shapes() +
                     acoustic_pipe_shapes() + acoustic_pcr_shapes() + acoustic_pipe_pcr_shapes();
    for (int cx = 0; cx < nvar; ++cx) {
      if (cx == acoustic_column_shapes() && !tma_ok_) continue;
      if (cx > acoustic_column_shapes() && !fused_usable(cx) && !chunked_usable(cx) &&
          !pipe_usable(cx) && !pcr_usable(cx) && !pipe_pcr_usable(cx))
        continue;
      // the parallel-solve variants agree with the others to rounding only:
      // the tuner picks them only where allowed (WFE_EXACT_COLUMN=0)
      if ((pcr_index(cx) >= 0 || pipe_pcr_index(cx) >= 0) && !pcr_allowed()) continue;
      float ms;
      tune_.column_cx = cx;
      if (time_ms([&] { return acoustic(N, X, (R)dt / (R)ns, 1, false); }, &ms)) return 1;
      if (ms < best) {
        best = ms;
        cached.column_cx = cx;
      }
    }
    launches_ = saved;
    CK(cudaStreamSynchronize(st_));
    CK(cudaGetLastError());
    cached.done = true;
    tune_ = cached;
    tune_store(key, tune_);
    return 0;
  }

  // --------------------------------------------------------------- pieces
  struct ProfRec {
    std::string name;
    cudaEvent_t e0, e1;
  };
  // Record mode (batched ensembles): a launch site appends its kind and
  // argument block to rec_ instead of launching.
  template <class A>
  bool record(int kind, const A& a) {
    if (!rec_) return false;
    Rec r;
    r.kind = kind;
    r.args.resize(sizeof(A));
    std::memcpy(r.args.data(), &a, sizeof(A));
    rec_->push_back(std::move(r));
    ++launches_;
    return true;
  }

  // wraps one launch: counted always, bracketed by events when profiling
  template <class F>
  void launch(const char* name, F&& f) {
    ProfRec r{name, nullptr, nullptr};
    if (profiling_) {  // inside a capture: recorded as event nodes of the graph
      cudaEventCreate(&r.e0);
      cudaEventCreate(&r.e1);
      cudaEventRecordWithFlags(r.e0, st_, cudaEventRecordExternal);
    }
    f();
    ++launches_;
    if (profiling_) {
      cudaEventRecordWithFlags(r.e1, st_, cudaEventRecordExternal);
      prof_.push_back(r);
    }
  }

  GhostJob<R> ghost_job(R** s, bool with_pip) {
    GhostJob<R> j{};
    auto add = [&](R* f, int kind) {
      j.f[j.n] = f;
      j.kind[j.n] = kind;
      ++j.n;
    };
    add(s[0], 1);
    add(s[1], 2);
    add(s[2], 3);
    add(s[3], 0);
    if (with_pip) add(s[4], 0);
    if (dp_.moisture) {
      add(s[5], 0);
      add(s[6], 0);
      add(s[7], 0);
    }
    return j;
  }

  TendArgs<R> tend_args(R** est, R dt) {
    TendArgs<R> a{};
    a.L = L_;
    a.b = db_;
    a.m = dm_;
    a.p = dp_;
    a.co = co_;
    a.dx = (R)g_.dx;
    a.dy = (R)g_.dy;
    a.dt = dt;
    a.u = est[0];
    a.v = est[1];
    a.w = est[2];
    a.thp = est[3];
    a.pip = est[4];
    a.qv = est[5];
    a.qc = est[6];
    a.qr = est[7];
    a.mfx = mfx_;
    a.mfy = mfy_;
    a.mfz = mfz_;
    a.clock = clock_;
    if (bdy_on_) {
      for (int v = 0; v < 5; ++v) {
        a.lo[v] = lo_[v];
        a.hi[v] = hi_[v];
      }
      a.wgt = wgt_;
    }
    return a;
  }

  // slow tendencies of est; moisture either into T_ (op) or into X as the
  // stage value N.q + dt_stage * tq
  void tendencies(R** est, R** N, R** X, R dt, R dt_stage, bool op) {
    if (!record(K_FLUX, FluxArgs<R>{L_, db_, dm_, est[0], est[1], est[2], mfx_, mfy_, mfz_}))
      launch("mass_flux", [&] { launch_mass_flux<R>(L_, db_, dm_, est[0], est[1], est[2], mfx_, mfy_, mfz_, st_); });
    TendArgs<R> a = tend_args(est, dt);
    if (dp_.moisture && dp_.pd_moist) {
      if (!record(K_PD, PdArgs<R>{a, ratio_[0], ratio_[1], ratio_[2]}))
        launch("pd_ratio", [&] { launch_pd_ratio<R>(a, ratio_[0], ratio_[1], ratio_[2], st_); });
      a.ratio_v = ratio_[0];
      a.ratio_c = ratio_[1];
      a.ratio_r = ratio_[2];
    }
    a.tu = T_[0];
    a.tv = T_[1];
    a.tw = T_[2];
    a.tth = T_[3];
    a.tpi = (op || bdy_on_) ? T_[4] : nullptr;
    a.tqv = T_[5];
    a.tqc = T_[6];
    a.tqr = T_[7];
    if (!op && dp_.moisture) {
      a.qn_v = N[5];
      a.qn_c = N[6];
      a.qn_r = N[7];
      a.qo_v = X[5];
      a.qo_c = X[6];
      a.qo_r = X[7];
      a.dt_stage = dt_stage;
    }
    if (!record(K_TEND, a)) {
      TendTmaParams<R> tp;
      if (tune_.tend_variant == 2 && tend_tma_usable() && tend_tma_params(a, &tp) == 0) {
        launch("tendencies", [&] {
          launch_tendencies<R>(a, 3, st_);
          launch_tend_scal_tma<R>(tp, st_);
        });
      } else {
        const int v = tune_.tend_variant == 1 ? 1 : (tune_.tend_variant == 3 ? 4 : 0);
        launch("tendencies", [&] { launch_tendencies<R>(a, v, st_); });
      }
    }
  }

  // The tuned forward u, v launch of one substep.
  int uv_launch(const AcouArgs<R>& a) {
    int rc = 0;
    if (uvp_ok_ && tune_.uv_variant == 1) {
      PipeUvParams<R> up;
      if (uv_pipe_params(a, &up)) return 1;
      launch("acoustic_uv", [&] { rc = launch_acoustic_uv_pipe<R>(up, st_); });
      if (rc) return fail("pipelined u, v launch");
    } else {
      launch("acoustic_uv", [&] { launch_acoustic_uv<R>(a, st_, tune_.uv_variant == 2 ? 1 : 0); });
    }
    return 0;
  }

  // The column launch of column variant v (a fused variant's own column
  // tile when the substep is not fused).
  int column_launch(const AcouArgs<R>& a, int v) {
    if (fused_usable(v)) v = acoustic_fused_column_shape(v - acoustic_column_shapes() - 1);
    int rc = 0;
    if (chunked_usable(v)) {
      const int f = chunked_index(v);
      launch("acoustic_column", [&] { rc = launch_acoustic_column_chunked<R>(a, f, st_); });
    } else if (pcr_usable(v)) {
      const int f = pcr_index(v);
      launch("acoustic_column", [&] { rc = launch_acoustic_column_pcr<R>(a, f, st_); });
    } else if (pipe_pcr_usable(v) &&
               acoustic_pipe_pcr_smem<R>(pipe_pcr_index(v), g_.nz, dp_.moisture != 0, a.tpi != nullptr,
                                         lvl_tab_ != nullptr) > 0) {
      const int f = pipe_pcr_index(v);
      PipeColParams<R> pp;
      if (pipe_params(a, f, &pp, true)) return 1;
      launch("acoustic_column", [&] { rc = launch_acoustic_column_pipe_pcr<R>(pp, f, st_); });
    } else if (pipe_usable(v) &&
               acoustic_pipe_smem<R>(pipe_index(v), g_.nz, dp_.moisture != 0, a.tpi != nullptr,
                                     lvl_tab_ != nullptr) > 0) {
      // (operator-level calls add the slow pi' tendency box: when that no
      // longer fits, the plain column kernel below takes the launch)
      const int f = pipe_index(v);
      PipeColParams<R> pp;
      if (pipe_params(a, f, &pp)) return 1;
      launch("acoustic_column", [&] { rc = launch_acoustic_column_pipe<R>(pp, f, st_); });
    } else if (tma_ok_ && v == acoustic_column_shapes()) {
      TmaColParams<R> tp;
      if (tma_params(a, &tp)) return 1;
      launch("acoustic_column", [&] { rc = launch_acoustic_column_tma<R>(tp, st_); });
    } else {
      launch("acoustic_column",
             [&] { rc = launch_acoustic_column<R>(a, v < acoustic_column_shapes() ? v : 0, st_); });
    }
    if (rc) return fail(rc == 2 ? "column too deep for the acoustic kernel" : "column kernel launch");
    return 0;
  }

  int replay_uv(const void* args) override { return uv_launch(*static_cast<const AcouArgs<R>*>(args)); }
  int replay_column(const void* args) override {
    return column_launch(*static_cast<const AcouArgs<R>*>(args), tune_.column_cx);
  }

  // ns acoustic substeps from time n (N) into the stage output X
  int acoustic(R** N, R** X, R dtau, int ns, bool op) {
    AcouArgs<R> a{};
    a.L = L_;
    a.b = db_;
    a.m = dm_;
    a.co = co_;
    a.p = dp_;
    a.dx = (R)g_.dx;
    a.dy = (R)g_.dy;
    a.dtau = dtau;
    a.n_pip = N[4];
    a.n_thp = N[3];
    a.qv = N[5];
    a.qc = N[6];
    a.qr = N[7];
    a.tu = T_[0];
    a.tv = T_[1];
    a.tw = T_[2];
    a.tth = T_[3];
    a.tpi = (op || bdy_on_) ? T_[4] : nullptr;
    R* pic[3] = {X[4], P1_, P2_};
    auto pbuf = [&](int t) -> R* {  // pi' after substep t-1 (t >= 1), time n for t <= 0
      if (t <= 0) return N[4];
      return pic[(ns - t) % 3];
    };
    const R* uin = N[0];
    const R* vin = N[1];
    // the fused kernel reads theta' of neighbouring columns that other CTAs
    // update: theta' alternates between X and a second buffer like u, v (the
    // last substep writes X); recorded launches keep the two-kernel form
    const bool fuse = !rec_ && fused_usable(tune_.column_cx);
    const R* thin = N[3];
    for (int t = 0; t < ns; ++t) {
      const bool last_parity = (ns - 1 - t) % 2 == 0;
      R* uout = last_parity ? X[0] : U2_;
      R* vout = last_parity ? X[1] : V2_;
      R* thout = (fuse && !last_parity) ? TH2_ : X[3];
      a.u_in = uin;
      a.v_in = vin;
      a.u_out = uout;
      a.v_out = vout;
      a.w_in = t == 0 ? N[2] : X[2];
      a.w_out = X[2];
      a.th_in = thin;
      a.th_out = thout;
      a.pi_prev = pbuf(t - 1);
      a.pi_cur = pbuf(t);
      a.pi_next = pbuf(t + 1);
      int rc = 0;
      if (fuse) {
        const int f = tune_.column_cx - acoustic_column_shapes() - 1;
        launch("acoustic_fused", [&] { rc = launch_acoustic_fused<R>(a, f, st_); });
      } else if (!record(K_UV, a)) {
        if (uv_launch(a)) return 1;
      }
      if (!fuse && !record(K_COL, a) && column_launch(a, tune_.column_cx)) return 1;
      if (rc) return fail(rc == 2 ? "column too deep for the acoustic kernel" : "fused substep launch");
      uin = uout;
      vin = vout;
      thin = thout;
      piprev_ = const_cast<R*>(a.pi_cur);
    }
    return 0;
  }

  // tensor map of a pitched field for box f of the TMA column kernel (cached)
  const CUtensorMap* tmap(const R* ptr, int f) {
    int bx, by;
    tma_col_box(f, &bx, &by);
    const auto key = std::make_pair(static_cast<const void*>(ptr), bx * 16 + by);
    auto it = tmaps_.find(key);
    if (it != tmaps_.end()) return &it->second;
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const cuuint64_t dims[3] = {(cuuint64_t)L_.px, (cuuint64_t)L_.py, (cuuint64_t)L_.pz};
    const cuuint64_t strides[2] = {(cuuint64_t)L_.px * sizeof(R), (cuuint64_t)L_.plane() * sizeof(R)};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)(g_.nz + 2)};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = tensor_map_encoder()(
        &m, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
        const_cast<R*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      fail("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
      return nullptr;
    }
    return &(tmaps_[key] = m);
  }

  bool tend_tma_usable() const { return tend_tma_ok_ && !(dp_.moisture && dp_.pd_moist); }

  // tensor map of a pitched field with box (bx, by, bz) (cached per pointer and box)
  const CUtensorMap* tmap3(const R* ptr, int bx, int by, int bz) {
    const auto key = std::make_pair(static_cast<const void*>(ptr), ((bx * 512) + by) * 512 + bz + 1000000000);
    auto it = tmaps_.find(key);
    if (it != tmaps_.end()) return &it->second;
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const cuuint64_t dims[3] = {(cuuint64_t)L_.px, (cuuint64_t)L_.py, (cuuint64_t)L_.pz};
    const cuuint64_t strides[2] = {(cuuint64_t)L_.px * sizeof(R), (cuuint64_t)L_.plane() * sizeof(R)};
    const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = tensor_map_encoder()(
        &m, sizeof(R) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3,
        const_cast<R*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
      fail("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
      return nullptr;
    }
    return &(tmaps_[key] = m);
  }

  int tend_tma_params(const TendArgs<R>& a, TendTmaParams<R>* tp) {
    std::memset(static_cast<void*>(tp), 0, sizeof(*tp));
    tp->a = a;
    tp->err = tma_err_;
    const CUtensorMap* m[3] = {tmap3(a.mfx, kTtX + 4, kTtY, kTtZ), tmap3(a.mfy, kTtX, kTtY + 1, kTtZ),
                               tmap3(a.mfz, kTtX, kTtY, kTtZ + 1)};
    for (auto* x : m)
      if (!x) return 1;
    tp->mfx = *m[0];
    tp->mfy = *m[1];
    tp->mfz = *m[2];
    const R* q[4] = {a.thp, a.qv, a.qc, a.qr};
    for (int f = 0; f < (dp_.moisture ? 4 : 1); ++f) {
      const CUtensorMap* x = tmap3(q[f], kTtX + 8, kTtY + 6, kTtZ + 6);
      if (!x) return 1;
      tp->q[f] = *x;
    }
    return 0;
  }

  int tma_params(const AcouArgs<R>& a, TmaColParams<R>* tp) {
    std::memset(static_cast<void*>(tp), 0, sizeof(*tp));
    tp->a = a;
    tp->err = tma_err_;
    tp->has_tpi = a.tpi != nullptr;
    const R* src[TC_N] = {a.u_out,  a.co.rtjx, a.v_out, a.co.rtjy, a.w_in,   a.pi_cur,
                          a.th_in,  a.tw,      a.tth,   a.tpi,     a.co.aw,  a.co.kt3,
                          a.b.thbw, a.b.dthbdz, a.qv,   a.qc,      a.qr,     a.b.qvb};
    for (int f = 0; f < TC_N; ++f) {
      if (f == TC_TPI && !a.tpi) continue;
      if (f >= TC_QV && !a.p.moisture) continue;
      const CUtensorMap* m = tmap(src[f], f);
      if (!m) return 1;
      tp->map[f] = *m;
    }
    return 0;
  }

  int uv_pipe_params(const AcouArgs<R>& a, PipeUvParams<R>* up) {
    std::memset(static_cast<void*>(up), 0, sizeof(*up));
    up->a = a;
    up->err = tma_err_;
    const R* src[UV_N] = {a.pi_cur, a.pi_prev, a.th_in, a.b.thb, a.qv, a.u_in, a.tu, a.v_in, a.tv};
    for (int f = 0; f < UV_N; ++f) {
      if (f == UV_QV && !a.p.moisture) continue;
      int bx, by, bz;
      uv_pipe_box(f, &bx, &by, &bz);
      const CUtensorMap* m = tmap3(src[f], bx, by, bz);
      if (!m) return 1;
      up->map[f] = *m;
    }
    return 0;
  }

  // pcr: the boxes of the pipelined parallel-solve shapes
  int pipe_params(const AcouArgs<R>& a, int shape, PipeColParams<R>* pp, bool pcr = false) {
    std::memset(static_cast<void*>(pp), 0, sizeof(*pp));
    pp->a = a;
    pp->err = tma_err_;
    pp->has_tpi = a.tpi != nullptr;
    pp->prof = lvl_tab_;
    const R* src[TC_N] = {a.u_out,  a.co.rtjx, a.v_out, a.co.rtjy, a.w_in,   a.pi_cur,
                          a.th_in,  a.tw,      a.tth,   a.tpi,     a.co.aw,  a.co.kt3,
                          a.b.thbw, a.b.dthbdz, a.qv,   a.qc,      a.qr,     a.b.qvb};
    for (int f = 0; f < TC_N; ++f) {
      if (f == TC_TPI && !a.tpi) continue;
      if (f >= TC_QV && !a.p.moisture) continue;
      if (pp->prof && pipe_prof_slot(f) >= 0) continue;
      int bx, by, bz;
      if (pcr)
        acoustic_pipe_pcr_box(shape, f, g_.nz, &bx, &by, &bz);
      else
        acoustic_pipe_box(shape, f, g_.nz, &bx, &by, &bz);
      const CUtensorMap* m = tmap3(src[f], bx, by, bz);
      if (!m) return 1;
      pp->map[f] = *m;
    }
    return 0;
  }

  int kessler(R** s, R dt) {
    KesArgs<R> k{L_, db_, dm_, dt, s[3], s[5], s[6], s[7], rain_, s[4]};
    int rc = 0;
    if (!record(K_KES, k)) launch("kessler", [&] { rc = launch_kessler<R>(k, st_); });
    if (rc) return fail("Kessler launch");
    return 0;
  }

  int surface(R** s, R dt) {
    SfcArgs<R> a{};
    a.L = L_;
    a.b = db_;
    a.m = dm_;
    a.dt = dt;
    a.start_hour = sf_.start_hour;
    a.doy = sf_.doy;
    a.nonlocal = sf_.nonlocal;
    a.clock = clock_;
    a.thp = s[3];
    a.qv = s[5];
    a.u = s[0];
    a.v = s[1];
    a.pip = s[4];
    a.qc = s[6];
    a.tsk = sf_.tsk;
    a.km = sf_.km;
    a.cdv = sf_.cdv;
    a.pblh = sf_.pblh;
    a.t2m = sf_.t2m;
    a.u10 = sf_.u10;
    a.soilt = sf_.soilt;
    a.tdeep = sf_.tdeep;
    a.land = sf_.land;
    a.lat = sf_.lat;
    a.lon = sf_.lon;
    a.soilw = sf_.soilw;
    a.scratch = sf_.scratch;
    int rc = 0;
    if (record(K_SFC, a)) {
      ++launches_;  // two kernels
      return 0;
    }
    launch("surface", [&] { rc = launch_sfc<R>(a, st_); });
    ++launches_;
    if (rc) return fail("surface physics launch");
    return 0;
  }

  // Integrator::step (src/dynamics/integrator.cpp:71-111) as launches on st_.
  int enqueue_step(R dt) {
    const int pN = perm_[0], pA = perm_[1], pB = perm_[2];
    const R stage_dt[3] = {dt / 3, dt / 2, dt};
    const int ns = hp_.acoustic_ns > 1 ? hp_.acoustic_ns : 1;
    const int nss[3] = {1, ns / 2 > 1 ? ns / 2 : 1, ns};
    R** N = S_[pN];
    for (int m = 0; m < 3; ++m) {
      R** est = m == 0 ? N : S_[m == 1 ? pA : pB];
      R** X = S_[m == 1 ? pB : pA];
      GhostJob<R> job = ghost_job(est, false);
      if (!record(K_FILL, FillArgs<R>{L_, job, dp_.bc_x_open, dp_.bc_y_open}))
        launch("fill_ghosts", [&] { launch_fill_ghosts<R>(L_, job, dp_.bc_x_open, dp_.bc_y_open, st_); });
      tendencies(est, N, X, dt, stage_dt[m], false);
      if (acoustic(N, X, stage_dt[m] / (R)nss[m], nss[m], false)) return 1;
    }
    R** Nn = S_[pA];
    if (dp_.moisture && dp_.microphysics && kessler(Nn, dt)) return 1;
    if (sfc_on_ && surface(Nn, dt)) return 1;
    advance_rotation();
    return 0;
  }

  void advance_rotation() {
    int p0 = perm_[0];
    perm_[0] = perm_[1];
    perm_[1] = perm_[2];
    perm_[2] = p0;
    phase_ = (phase_ + 1) % 3;
  }

  // --------------------------------------------------------------- memory
  // When every column of the run-constant column coefficients (the
  // reference's rtjx, rtjy, aw, kt3, theta_b^w, dtheta_b/dz, qv_b) holds the
  // same values level by level -- flat ground and a uniform map factor --
  // the pipelined column kernels read them from per-level tables
  // (the values of column (0, 0)) instead of streaming a box of each per
  // tile: the same values, bit for bit.  Checked over the points the column
  // kernel reads.  Likewise the base state's thb, pib, rhob and rhobw for
  // the mass-flux, Kessler and u, v kernels (DBase::lvl), checked over every
  // column they read (the interior and its three-wide ring) at levels
  // 0 .. nz.  WFE_LEVEL_TABLES=0 keeps the 3D fields.
  int level_tables() {
    const char* e = std::getenv("WFE_LEVEL_TABLES");
    if (e && e[0] == '0') return 0;
    if (base_tables()) return 1;
    const int nx = g_.nx, ny = g_.ny, nz = g_.nz, n1 = nz + 1;
    const R* src[PF_N] = {rtjx_, rtjy_, aw_, kt3_, db_.thbw, db_.dthbdz, db_.qvb};
    std::vector<R> host(L_.n3()), tab((size_t)PF_N * n1);
    for (int q = 0; q < PF_N; ++q) {
      if (q == PF_QVB && !dp_.moisture) continue;
      CK(cudaMemcpy(host.data(), src[q], L_.n3() * sizeof(R), cudaMemcpyDeviceToHost));
      const int ilast = q == PF_RTJX ? nx : nx - 1, jlast = q == PF_RTJY ? ny : ny - 1;
      for (int k = 0; k < n1; ++k) {
        const R v = host[L_.at(0, 0, k)];
        tab[(size_t)q * n1 + k] = v;
        if (k == nz) continue;  // the kernel reads levels 0 .. nz-1
        for (int j = 0; j <= jlast; ++j)
          for (int i = 0; i <= ilast; ++i)
            if (std::memcmp(&host[L_.at(i, j, k)], &v, sizeof(R)) != 0) return 0;
      }
    }
    if (!(lvl_tab_ = alloc(tab.size()))) return 1;
    CK(cudaMemcpy(lvl_tab_, tab.data(), tab.size() * sizeof(R), cudaMemcpyHostToDevice));
    return 0;
  }

  int base_tables() {
    const int nx = g_.nx, ny = g_.ny, nz = g_.nz, pz = L_.pz;
    const R* src[BL_N] = {db_.thb, db_.pib, db_.rhob, db_.rhobw};
    std::vector<R> host(L_.n3()), tab((size_t)BL_N * pz);
    for (int q = 0; q < BL_N; ++q) {
      CK(cudaMemcpy(host.data(), src[q], L_.n3() * sizeof(R), cudaMemcpyDeviceToHost));
      for (int k = -kOZ; k < pz - kOZ; ++k) {
        const R v = host[L_.at(0, 0, k)];
        tab[(size_t)q * pz + L_.at1(k)] = v;
        if (k < 0 || k > nz) continue;
        for (int j = -kRefNG; j < ny + kRefNG; ++j)
          for (int i = -kRefNG; i < nx + kRefNG; ++i)
            if (std::memcmp(&host[L_.at(i, j, k)], &v, sizeof(R)) != 0) return 0;
      }
    }
    R* d = alloc(tab.size());
    if (!d) return 1;
    CK(cudaMemcpy(d, tab.data(), tab.size() * sizeof(R), cudaMemcpyHostToDevice));
    db_.lvl = d;
    return 0;
  }

  R* alloc(size_t n) {
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, n * sizeof(R));
    if (e != cudaSuccess) {
      fail(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return nullptr;
    }
    cudaMemset(p, 0, n * sizeof(R));
    allocs_.push_back(p);
    return (R*)p;
  }

  // reference padded layout -> pitched; columns/rows outside the reference's
  // padded range replicate the nearest one so that no padding is uninitialised
  void to_pitched(const double* ref, R* out, bool replicate) {
    for (int k = -kOZ; k < L_.pz - kOZ; ++k)
      for (int j = -kOY; j < L_.py - kOY; ++j) {
        const double* row = ref + g_.idx(-3, j, k);
        R* o = out + L_.at(-kOX, j, k);
        for (int i = -kOX; i < L_.px - kOX; ++i) {
          int ic = i < -3 ? -3 : (i > g_.nx + 2 ? g_.nx + 2 : i);
          o[i + kOX] = (R)row[ic + 3];
        }
      }
    (void)replicate;
  }

  void from_pitched(const R* in, double* ref) {
    for (int k = -3; k < g_.nz + 4; ++k)
      for (int j = -3; j < g_.ny + 3; ++j)
        for (int i = -3; i < g_.nx + 3; ++i) ref[g_.idx(i, j, k)] = (double)in[L_.at(i, j, k)];
  }

  // put3d / put2d / put1d overwrite buffers that queued steps may still read
  // (boundary targets switched between runs, surface fields): the model's
  // stream is drained first (the copies themselves are not stream-ordered,
  // and an ensemble orders its members' streams after its own work)
  int put3d(R* d, const std::vector<double>& ref) {
    to_pitched(ref.data(), stage_tmp(L_.n3()), true);
    CK(cudaStreamSynchronize(st_));
    CK(cudaMemcpy(d, tmp_.data(), L_.n3() * sizeof(R), cudaMemcpyHostToDevice));
    return 0;
  }
  int put2d(R* d, const std::vector<double>& ref2) {
    CK(cudaStreamSynchronize(st_));
    R* o = stage_tmp(L_.n2());
    for (int j = -kOY; j < L_.py - kOY; ++j)
      for (int i = -kOX; i < L_.px - kOX; ++i) {
        int ic = i < -3 ? -3 : (i > g_.nx + 2 ? g_.nx + 2 : i);
        o[L_.at2(i, j)] = (R)ref2[g_.idx2(ic, j)];
      }
    CK(cudaMemcpy(d, o, L_.n2() * sizeof(R), cudaMemcpyHostToDevice));
    return 0;
  }
  int put1d(R* d, const std::vector<double>& v) {
    CK(cudaStreamSynchronize(st_));
    R* o = stage_tmp(L_.pz);
    for (int q = 0; q < L_.pz; ++q) o[q] = (R)v[q];
    CK(cudaMemcpy(d, o, L_.pz * sizeof(R), cudaMemcpyHostToDevice));
    return 0;
  }
  R* stage_tmp(size_t n) {
    if (tmp_.size() < n) tmp_.resize(n);
    return tmp_.data();
  }

  int fail(const std::string& m) {
    err_ = m;
    return 1;
  }

  void release() {
    for (auto& ge : gexec_)
      if (ge) cudaGraphExecDestroy(ge);
    for (void* p : allocs_) cudaFree(p);
    allocs_.clear();
    if (clock_) cudaFree(clock_);
    if (wd_) cudaFree(wd_);
    if (mass_planes_) cudaFree(mass_planes_);
    if (mass_) cudaFree(mass_);
    if (tma_err_) cudaFree(tma_err_);
    tma_err_ = nullptr;
    if (stage_) cudaFreeHost(stage_);
    if (cs_st_) {
      cudaStreamSynchronize(cs_st_);
      cudaStreamDestroy(cs_st_);
    }
    if (snap_ev_) cudaEventDestroy(snap_ev_);
    if (snap_buf_) cudaFree(snap_buf_);
    if (up_buf_) cudaFree(up_buf_);
    up_buf_ = nullptr;
    up_cap_ = 0;
    cs_st_ = nullptr;
    snap_ev_ = nullptr;
    snap_buf_ = nullptr;
    if (st_) cudaStreamDestroy(st_);
    clock_ = nullptr;
    wd_ = nullptr;
    if (wd_async_) cudaFree(wd_async_);
    wd_async_ = nullptr;
    if (wd_host_) cudaFreeHost(wd_host_);
    wd_host_ = nullptr;
    for (auto& e : wd_ev_)
      if (e) {
        cudaEventDestroy(e);
        e = nullptr;
      }
    mass_planes_ = nullptr;
    mass_ = nullptr;
    stage_ = nullptr;
    st_ = nullptr;
  }

  struct SfcBufs {
    R *tsk = nullptr, *tdeep = nullptr, *land = nullptr, *lat = nullptr, *lon = nullptr,
      *soilw = nullptr, *cdv = nullptr, *pblh = nullptr, *t2m = nullptr, *u10 = nullptr,
      *km = nullptr, *soilt = nullptr, *scratch = nullptr;
    double start_hour = 0;
    int doy = 1;
    bool nonlocal = false;
  };

  const CaseSetup* cs_ = nullptr;
  RefGrid g_{};
  HostParams hp_{};
  Layout L_{};
  int dev_ = 0;
  cudaStream_t st_ = nullptr;
  DMetric<R> dm_{};
  DBase<R> db_{};
  DCoef<R> co_{};
  DParams<R> dp_{};
  R* S_[3][8] = {};
  R* T_[8] = {};
  R *mfx_ = nullptr, *mfy_ = nullptr, *mfz_ = nullptr;
  R *U2_ = nullptr, *V2_ = nullptr, *P1_ = nullptr, *P2_ = nullptr, *TH2_ = nullptr;
  R* ratio_[3] = {};
  R *rtjx_ = nullptr, *rtjy_ = nullptr, *kt3_ = nullptr, *aw_ = nullptr;
  R* rain_ = nullptr;
  R* piprev_ = nullptr;
  R* lo_[5] = {};
  R* hi_[5] = {};
  R* wgt_ = nullptr;
  bool bdy_on_ = false, sfc_on_ = false;
  double t_lo_ = 0, t_hi_ = 0;
  SfcBufs sf_;
  double* clock_ = nullptr;
  unsigned int* wd_ = nullptr;
  unsigned int* wd_async_ = nullptr;   // two watchdog slots (absmax_begin / end)
  unsigned int* wd_host_ = nullptr;    // mapped page-locked results, one per slot
  unsigned int* wd_host_dev_ = nullptr;  // the same words as the device sees them
  cudaEvent_t wd_ev_[2] = {nullptr, nullptr};
  double *mass_planes_ = nullptr, *mass_ = nullptr;
  R* stage_ = nullptr;
  std::vector<R> tmp_;
  std::vector<void*> allocs_;
  int perm_[3] = {0, 1, 2};
  int phase_ = 0;
  cudaGraphExec_t gexec_[3] = {nullptr, nullptr, nullptr};
  bool graphs_valid_ = false;
  long gen_ = 0;  // changes whenever buffer roles or physics switches change
  std::vector<Rec>* rec_ = nullptr;  // record mode when set
  bool tma_ok_ = false;              // TMA column variant usable
  bool fused_ok_ = false;            // fused substep kernels prepared
  bool pipe_ok_ = false;             // pipelined column kernels prepared
  bool uvp_ok_ = false;              // pipelined u, v kernel prepared
  bool tend_tma_ok_ = false;         // TMA-staged scalar tendencies usable
  R* lvl_tab_ = nullptr;             // the column coefficients' level tables (PF_*), or null
  unsigned* tma_err_ = nullptr;      // set by a TMA tile load that timed out
  std::map<std::pair<const void*, int>, CUtensorMap> tmaps_;
  cudaStream_t cs_st_ = nullptr;     // snapshot copy stream
  cudaEvent_t snap_ev_ = nullptr;
  void* snap_buf_ = nullptr;         // packed snapshot staging
  void* up_buf_ = nullptr;           // interior upload staging
  size_t up_cap_ = 0;
  size_t snap_cap_ = 0;
  std::function<void*(const void*)> lin_map_;
  double graph_dt_ = 0;
  long launches_ = 0, glaunches_ = 0;
  bool profiling_ = false;
  std::vector<ProfRec> prof_;
  Tune tune_;
};

// --------------------------------------------------------------- ensembles
template <typename R>
class EnsembleT final : public Ensemble {
 public:
  ~EnsembleT() override { release(); }

  int init(const std::vector<ModelT<R>*>& m) {
    mem_ = m;
    if (mem_.empty()) return fail("an ensemble needs at least one member");
    dev_ = mem_[0]->device();
    const std::string sig = mem_[0]->batch_signature();
    for (auto* x : mem_) {
      if (x->device() != dev_) return fail("ensemble members must share one device");
      if (x->batch_signature() != sig)
        return fail("ensemble members must share moisture, microphysics, positive-definite "
                    "moisture, boundary, surface-physics and substep settings");
      if (x->phase() != mem_[0]->phase())
        return fail("ensemble members must be at the same step phase");
      nz_max_ = std::max(nz_max_, x->layout().nz);
    }
    CK(cudaSetDevice(dev_));
    CK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&ev_, cudaEventDisableTiming));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_));
    sms_ = sms;
    if (prepare_acoustic_column<R>(nz_max_) || prepare_kessler<R>(nz_max_) || prepare_sfc<R>(nz_max_))
      return fail("nz too large for the column kernels' shared memory");
    if (sfc_needs_scratch<R>(nz_max_))
      for (auto* x : mem_)
        if (x->ensure_sfc_scratch()) return fail(x->error());
    gens_.assign(mem_.size(), -1);
    return 0;
  }

  // steps the first run takes to pick the mode (it needs at least this many)
  static constexpr int kModePickSteps = 19;

  int run(int nsteps, double dt, double t0) override {
    CK(cudaSetDevice(dev_));
    if (begin(dt)) return 1;
    for (auto* x : mem_) launch_clock(x->clock_ptr(), t0, x->bdy_t_lo(), x->bdy_t_hi(), dt, 0, st_);
    int s = 0;
    // "members" | "sequential" | "batched": no timing
    const char* em = std::getenv("WFE_ENSEMBLE_MODE");
    if (em && *em) {
      mode_done_ = true;
      const std::string m(em);
      tune_.persist = m == "members" ? 2 : (m == "sequential" ? 3 : ((tune_.persist & 1) | 4));
    }
    if (!mode_done_ && nsteps >= kModePickSteps) {
      // pick on real steps among the batched launches, the members' own
      // graphs on concurrent streams and the members' own graphs one after
      // another (all three give the same values, bit for bit): three warm-up
      // steps of each mode capture every phase's graphs; then the batched
      // mode is timed over two steps and the two close modes over four, in
      // the order concurrent, sequential, sequential, concurrent, so that a
      // step cost that drifts as the flow develops weighs on both alike
      float tb = 0, tc = 0, tq = 0, t1 = 0, t2 = 0;
      if (batched_steps(3, dt) || timed([&] { return batched_steps(2, dt); }, &tb)) return 1;
      if (member_steps(3, dt, false) || member_steps(3, dt, true)) return 1;
      if (timed([&] { return member_steps(2, dt, false); }, &t1)) return 1;
      if (timed([&] { return member_steps(2, dt, true); }, &t2)) return 1;
      tq = t2;
      if (timed([&] { return member_steps(2, dt, true); }, &t2)) return 1;
      tq += t2;
      if (timed([&] { return member_steps(2, dt, false); }, &t2)) return 1;
      tc = t1 + t2;
      tb *= 2;  // per four steps, as tc and tq
      s = kModePickSteps;
      mode_done_ = true;
      if (tc <= tb && tc <= tq) tune_.persist = 2;
      else if (tq <= tb) tune_.persist = 3;
      else tune_.persist = (tune_.persist & 1) | 4;
      tune_store(tune_key(), tune_);
    }
    if (tune_.persist == 2 || tune_.persist == 3) {
      if (member_steps(nsteps - s, dt, tune_.persist == 3)) return 1;
      return 0;
    }
    if (batched_steps(nsteps - s, dt)) return 1;
    return finish();
  }

  // members' own graphs, each on its own stream, ordered after the ensemble
  // stream's work, and the ensemble stream after them: interleaved step by
  // step so that the members run concurrently, or (sequential) each member's
  // steps after the previous member's, as a serial run of the members does
  int member_steps(int nsteps, double dt, bool sequential) {
    CK(cudaEventRecord(ev_, st_));
    for (auto* x : mem_) {
      CK(cudaStreamWaitEvent(x->stream(), ev_, 0));
      if (x->tune_for(dt)) return fail(x->error());
    }
    if (sequential) {
      for (size_t q = 0; q < mem_.size(); ++q) {
        if (q > 0) {
          CK(cudaEventRecord(ev_, mem_[q - 1]->stream()));
          CK(cudaStreamWaitEvent(mem_[q]->stream(), ev_, 0));
        }
        if (mem_[q]->graph_steps(nsteps, dt)) return fail(mem_[q]->error());
      }
    } else {
      for (int s = 0; s < nsteps; ++s)
        for (auto* x : mem_)
          if (x->graph_steps(1, dt)) return fail(x->error());
    }
    long l = 0;
    for (auto* x : mem_) {
      CK(cudaEventRecord(ev_, x->stream()));
      CK(cudaStreamWaitEvent(st_, ev_, 0));
      l += x->launches_per_step();
    }
    if (tune_.persist == 2 || tune_.persist == 3) launches_ = l;
    return 0;
  }

  template <typename F>
  int timed(F&& f, float* ms) {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    CK(cudaEventRecord(e0, st_));
    int rc = f();
    CK(cudaEventRecord(e1, st_));
    CK(cudaEventSynchronize(e1));
    CK(cudaEventElapsedTime(ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
  }

  int batched_steps(int nsteps, double dt) {
    for (int s = 0; s < nsteps; ++s) {
      Phase& P = ph_[mem_[0]->phase()];
      if (!P.ge) {
        if (build(P, dt)) return 1;
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        int rc = issue(P, (int)P.pos.size());
        cudaError_t ce = cudaStreamEndCapture(st_, &gr);
        if (rc) return 1;
        if (ce != cudaSuccess) return fail(std::string("graph capture: ") + cudaGetErrorString(ce));
        CK(cudaGraphInstantiate(&P.ge, gr, 0));
        cudaGraphDestroy(gr);
      }
      CK(cudaGraphLaunch(P.ge, st_));
      for (auto* x : mem_) x->rotate();
    }
    return 0;
  }

  int step(double dt, double t) override {
    CK(cudaSetDevice(dev_));
    if (begin(dt)) return 1;
    for (auto* x : mem_) launch_clock(x->clock_ptr(), t, x->bdy_t_lo(), x->bdy_t_hi(), dt, 0, st_);
    Phase& P = ph_[mem_[0]->phase()];
    if (!P.built && build(P, dt)) return 1;
    if (issue(P, (int)P.pos.size())) return 1;
    for (auto* x : mem_) x->rotate();
    if (finish()) return 1;
    return sync();
  }

  int sync() override {
    CK(cudaStreamSynchronize(st_));
    CK(cudaGetLastError());
    return 0;
  }

  int time_run(int nsteps, double dt, double t0, double* ms) override {
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    if (begin(dt)) return 1;  // tuning and member ordering outside the timed region
    CK(cudaEventRecord(e0, st_));
    int rc = run(nsteps, dt, t0);
    CK(cudaEventRecord(e1, st_));
    CK(cudaEventSynchronize(e1));
    float f = 0;
    CK(cudaEventElapsedTime(&f, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = f;
    return rc;
  }

  long launches_per_step() const override { return launches_; }
  void variants(int* tend, int* column, int* persist) const override {
    *tend = tune_.tend_variant;
    *column = tune_.column_cx;
    *persist = (tune_.persist & 4) ? (tune_.persist & 1) : tune_.persist;
  }

 private:
  // tune_.persist: bit 0 the persistent grid of the batched launches, 4 the
  // batched mode chosen on real steps; 2 the members' own graphs chosen
  bool mode_done_ = false;  // batched vs members' own graphs decided
  struct Work {
    int4* d = nullptr;
    int n = 0;
  };
  struct Pos {
    int kind;
    size_t off;                // member argument blocks at arena + off
    std::vector<Work*> subs;   // work list of each sub-launch
  };
  struct Phase {
    std::vector<Pos> pos;
    unsigned char* d_args = nullptr;
    size_t cap = 0;
    cudaGraphExec_t ge = nullptr;
    bool built = false;
  };

  int variant_of(int kind) const {
    return kind == K_TEND ? tune_.tend_variant : (kind == K_COL ? tune_.column_cx : 0);
  }

  // Orders the ensemble stream after the members' streams, tunes once and
  // drops phases whose members changed buffers or whose dt changed.
  int begin(double dt) {
    for (auto* x : mem_) {
      CK(cudaEventRecord(ev_, x->stream()));
      CK(cudaStreamWaitEvent(st_, ev_, 0));
    }
    bool stale = dt != dt_;
    for (size_t m = 0; m < mem_.size(); ++m)
      if (gens_[m] != mem_[m]->generation()) stale = true;
    if (stale) {
      for (auto& P : ph_) drop(P);
      for (size_t m = 0; m < mem_.size(); ++m) gens_[m] = mem_[m]->generation();
      dt_ = dt;
    }
    return autotune(dt);
  }

  // Orders the members' streams after the ensemble's work.
  int finish() {
    CK(cudaEventRecord(ev_, st_));
    for (auto* x : mem_) CK(cudaStreamWaitEvent(x->stream(), ev_, 0));
    CK(cudaGetLastError());
    return 0;
  }

  void drop(Phase& P) {
    if (P.ge) cudaGraphExecDestroy(P.ge);
    P.ge = nullptr;
    P.built = false;
    P.pos.clear();
  }

  // Records every member's step from the current phase, checks that the
  // launch sequences agree, uploads the argument blocks and builds the work
  // lists for the current variants.
  int build(Phase& P, double dt) {
    const size_t M = mem_.size();
    std::vector<std::vector<Rec>> recs(M);
    for (size_t m = 0; m < M; ++m) {
      if (mem_[m]->record_step(dt, &recs[m])) return fail(mem_[m]->error());
      Rec c;
      c.kind = K_CLOCK;
      ClockArgs ca{mem_[m]->clock_ptr(), 0, 0, 0, 0, 1};
      c.args.resize(sizeof(ca));
      std::memcpy(c.args.data(), &ca, sizeof(ca));
      recs[m].push_back(std::move(c));
    }
    const size_t n = recs[0].size();
    for (size_t m = 1; m < M; ++m) {
      if (recs[m].size() != n) return fail("ensemble members record different steps");
      for (size_t p = 0; p < n; ++p)
        if (recs[m][p].kind != recs[0][p].kind) return fail("ensemble members record different steps");
    }
    P.pos.clear();
    size_t total = 0;
    for (size_t p = 0; p < n; ++p) {
      const size_t sz = kind_args_size<R>(recs[0][p].kind);
      P.pos.push_back(Pos{recs[0][p].kind, total, {}});
      total += (M * sz + 255) / 256 * 256;
    }
    std::vector<unsigned char> host(total);
    for (size_t p = 0; p < n; ++p) {
      const size_t sz = kind_args_size<R>(P.pos[p].kind);
      for (size_t m = 0; m < M; ++m) {
        if (recs[m][p].args.size() != sz) return fail("argument block size mismatch");
        std::memcpy(host.data() + P.pos[p].off + m * sz, recs[m][p].args.data(), sz);
      }
      const int kind = P.pos[p].kind, var = variant_of(kind);
      for (int sub = 0; sub < kind_subs<R>(kind, var); ++sub) {
        std::vector<const void*> args(M);
        for (size_t m = 0; m < M; ++m) args[m] = recs[m][p].args.data();
        Work* w = work_for(kind, var, sub, args);
        if (!w) return 1;
        P.pos[p].subs.push_back(w);
      }
    }
    if (P.cap < total) {
      if (P.d_args) cudaFree(P.d_args);
      P.d_args = nullptr;
      P.cap = 0;
      CK(cudaMalloc(&P.d_args, total));
      P.cap = total;
    }
    CK(cudaMemcpyAsync(P.d_args, host.data(), total, cudaMemcpyHostToDevice, st_));
    CK(cudaStreamSynchronize(st_));
    long l = 0;
    for (auto& q : P.pos) l += (long)q.subs.size();
    launches_ = l;
    P.built = true;
    return 0;
  }

  // work list of one sub-launch over all members, shared by every position
  // with the same kind, variant and member grids
  Work* work_for(int kind, int var, int sub, const std::vector<const void*>& args) {
    std::ostringstream key;
    key << kind << "/" << var << "/" << sub;
    std::vector<dim3> grids(args.size());
    for (size_t m = 0; m < args.size(); ++m) {
      grids[m] = kind_grid<R>(kind, var, sub, args[m], nz_max_);
      key << "|" << grids[m].x << "x" << grids[m].y << "x" << grids[m].z;
    }
    auto it = work_.find(key.str());
    if (it != work_.end()) return &it->second;
    std::vector<int4> items;
    for (size_t m = 0; m < args.size(); ++m)
      for (unsigned z = 0; z < grids[m].z; ++z)
        for (unsigned y = 0; y < grids[m].y; ++y)
          for (unsigned x = 0; x < grids[m].x; ++x)
            items.push_back(make_int4((int)m, (int)x, (int)y, (int)z));
    Work w;
    w.n = (int)items.size();
    if (w.n > 0) {
      cudaError_t e = cudaMalloc(&w.d, items.size() * sizeof(int4));
      if (e == cudaSuccess)
        e = cudaMemcpy(w.d, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        fail(std::string("work list: ") + cudaGetErrorString(e));
        return nullptr;
      }
    }
    return &(work_[key.str()] = w);
  }

  // issues the first npos positions of a built phase on st_
  int issue(const Phase& P, int npos) {
    for (int p = 0; p < npos; ++p) {
      const Pos& q = P.pos[p];
      const int var = variant_of(q.kind);
      for (int sub = 0; sub < (int)q.subs.size(); ++sub) {
        const Work* w = q.subs[sub];
        int nblocks = w->n;
        if (tune_.persist & 1) {
          int occ = kind_occupancy<R>(q.kind, var, sub, nz_max_);
          nblocks = std::min(w->n, occ * sms_);
        }
        if (launch_kind_batch<R>(q.kind, var, sub, P.d_args + q.off, w->d, w->n, nblocks, nz_max_,
                                 st_))
          return fail("batched launch: tile shape does not fit the deepest member");
      }
    }
    CK(cudaGetLastError());
    return 0;
  }

  std::string tune_key() const {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, dev_);
    std::ostringstream k;
    std::string name = prop.name;
    for (char& ch : name)
      if (ch == ' ') ch = '_';
    k << "ens2|" << name << "|" << (sizeof(R) * 8) << "|" << mem_[0]->batch_signature();
    for (auto* x : mem_) k << "|" << x->layout().nx << "x" << x->layout().ny << "x" << x->layout().nz;
    return k.str();
  }

  // Times the variants on the first stage's launches up to its acoustic
  // column (they read time n and write only scratch, tendencies and the
  // stage output, which the step overwrites).  WFE_TUNE=0 keeps defaults.
  int autotune(double dt) {
    if (tune_.done) return 0;
    tune_.done = true;
    const char* env = std::getenv("WFE_TUNE");
    if (env && env[0] == '0') return 0;
    const std::string key = tune_key();
    Tune cached;
    if (tune_lookup(key, &cached)) {
      tune_ = cached;
      mode_done_ = tune_.persist == 2 || tune_.persist == 3 || (tune_.persist & 4);
      return 0;
    }
    int upto = -1;
    auto stage0 = [&](float* ms) -> int {
      Phase T;
      if (build(T, dt)) return 1;
      if (upto < 0)
        for (int p = 0; p < (int)T.pos.size() && upto < 0; ++p)
          if (T.pos[p].kind == K_COL) upto = p + 1;
      cudaEvent_t e0, e1;
      CK(cudaEventCreate(&e0));
      CK(cudaEventCreate(&e1));
      *ms = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        CK(cudaEventRecord(e0, st_));
        if (issue(T, upto)) return 1;
        CK(cudaEventRecord(e1, st_));
        CK(cudaEventSynchronize(e1));
        float f = 0;
        CK(cudaEventElapsedTime(&f, e0, e1));
        *ms = std::min(*ms, f);
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (T.d_args) cudaFree(T.d_args);
      return 0;
    };
    Tune best = tune_;
    float bt = 1e30f, ms;
    for (int v = 0; v < 2; ++v) {
      tune_.tend_variant = v;
      if (stage0(&ms)) return 1;
      if (ms < bt) bt = ms, best.tend_variant = v;
    }
    tune_.tend_variant = best.tend_variant;
    bt = 1e30f;
    for (int c = 0; c < acoustic_column_shapes(); ++c) {
      if (!acoustic_column_fits<R>(nz_max_, c)) continue;
      tune_.column_cx = c;
      if (stage0(&ms)) return 1;
      if (ms < bt) bt = ms, best.column_cx = c;
    }
    tune_.column_cx = best.column_cx;
    bt = 1e30f;
    for (int pz = 0; pz < 2; ++pz) {
      tune_.persist = pz;
      if (stage0(&ms)) return 1;
      if (ms < bt) bt = ms, best.persist = pz;
    }
    CK(cudaStreamSynchronize(st_));
    best.done = true;
    tune_ = best;
    tune_store(key, tune_);
    return 0;
  }

  int fail(const std::string& m) {
    err_ = m;
    return 1;
  }

  void release() {
    for (auto& P : ph_) {
      drop(P);
      if (P.d_args) cudaFree(P.d_args);
      P.d_args = nullptr;
    }
    for (auto& kv : work_)
      if (kv.second.d) cudaFree(kv.second.d);
    work_.clear();
    if (ev_) cudaEventDestroy(ev_);
    if (st_) cudaStreamDestroy(st_);
    ev_ = nullptr;
    st_ = nullptr;
  }

  std::vector<ModelT<R>*> mem_;
  std::vector<long> gens_;
  int dev_ = 0, sms_ = 148, nz_max_ = 0;
  cudaStream_t st_ = nullptr;
  cudaEvent_t ev_ = nullptr;
  Phase ph_[3];
  std::map<std::string, Work> work_;
  Tune tune_;
  double dt_ = -1;
  long launches_ = 0;
};

Ensemble* Ensemble::create(const std::vector<Model*>& members, std::string* err) {
  if (members.empty()) {
    *err = "an ensemble needs at least one member";
    return nullptr;
  }
  const bool f64 = members[0]->fp64();
  for (Model* m : members)
    if (!m || m->fp64() != f64) {
      *err = "ensemble members must share one precision";
      return nullptr;
    }
  Ensemble* e = nullptr;
  int rc;
  if (f64) {
    std::vector<ModelT<double>*> v;
    for (Model* m : members) v.push_back(static_cast<ModelT<double>*>(m));
    auto* t = new EnsembleT<double>();
    rc = t->init(v);
    e = t;
  } else {
    std::vector<ModelT<float>*> v;
    for (Model* m : members) v.push_back(static_cast<ModelT<float>*>(m));
    auto* t = new EnsembleT<float>();
    rc = t->init(v);
    e = t;
  }
  if (rc) {
    *err = e->error();
    delete e;
    return nullptr;
  }
  return e;
}

Model* Model::create(const CaseSetup& cs, bool fp64, int device, std::string* err) {
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    *err = std::string("no CUDA device available: ") + cudaGetErrorString(e);
    return nullptr;
  }
  if (device < 0 || device >= ndev) {
    *err = "device index out of range";
    return nullptr;
  }
  Model* m = nullptr;
  int rc;
  if (fp64) {
    auto* t = new ModelT<double>();
    rc = t->init(cs, device);
    m = t;
  } else {
    auto* t = new ModelT<float>();
    rc = t->init(cs, device);
    m = t;
  }
  if (rc) {
    *err = m->error();
    delete m;
    return nullptr;
  }
  return m;
}

}  // namespace wfe
