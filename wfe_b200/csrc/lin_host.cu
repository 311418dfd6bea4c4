// Tangent-linear and adjoint runs of the model step (Lin, model.hpp): the
// dynamics with moisture and the Kessler column.
//
// The step is taken from the model's own recorded launch sequence, so the
// linearised runs follow the forward's buffer rotation exactly: every
// state-like forward buffer has a linearised mirror, and each recorded
// argument block is translated to the mirrors to drive the TL / AD kernel of
// that launch (lin.cu).
//
// TL:  per launch, the TL kernel (forward values still in place) and then the
//      forward launch; the column's TL launch writes the forward column's
//      outputs itself, bit for bit.
// AD:  the forward pass (the model's own graphs) stores the time-n state at
//      the start of every segment of `every` steps (the last segment is not
//      run there: its replay below is its forward run).  The reverse sweep
//      takes the segments last to first: it restores the segment's start
//      state, replays the segment forward with one graph that saves every
//      buffer each launch overwrites (an undo log), and walks the launches
//      backwards with a second graph: restore the launch's outputs from the
//      log, run its AD kernel -- except the acoustic column, whose adjoint
//      runs first and reads the forward solution from the outputs still in
//      place (its inputs updated in place from the log).  A step is a
//      function of its time-n state alone (every other buffer is written
//      before it is read), so restoring that state reproduces the segment.
// Cost per step: the forward pass (all segments but the last), the replay,
// the undo-log copies and the AD kernels.
#include <cuda_runtime.h>

#include <cstring>
#include <initializer_list>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "model.hpp"

namespace wfe {
namespace {

#define LCK(call)                                                                 \
  do {                                                                            \
    cudaError_t e__ = (call);                                                     \
    if (e__ != cudaSuccess) return fail(std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

template <typename R>
class LinT final : public Lin {
 public:
  ~LinT() override { release(); }

  int init(Model* m) {
    m_ = m;
    std::string why;
    if (!m->linearisable(&why)) return fail(why);
    st_ = static_cast<cudaStream_t>(m->stream_handle());
    for (auto& b : m->state_buffers()) {
      void* p = nullptr;
      LCK(cudaMalloc(&p, b.second * sizeof(R)));
      LCK(cudaMemsetAsync(p, 0, b.second * sizeof(R), st_));
      map_[b.first] = p;
      bufs_.push_back({static_cast<R*>(p), b.second});
      fwd_.push_back({static_cast<R*>(b.first), b.second});
    }
    n3_ = bufs_.empty() ? 0 : bufs_[0].second;
    for (R*& f : scr_.f) {
      LCK(cudaMalloc(&f, n3_ * sizeof(R)));
      LCK(cudaMemsetAsync(f, 0, n3_ * sizeof(R), st_));
    }
    std::vector<Rec> recs;
    if (m->record_step(1.0, &recs)) return fail(m->error());
    learn_layout(recs);
    const int pr = lin_prepare<R>(L_.nz);
    if (pr == 2) return fail("column deeper than the linearised kernels hold");
    if (pr) return fail("linearised column kernels: shared memory limit");
    m->set_lin_map([this](const void* p) -> void* {
      auto it = map_.find(p);
      return it == map_.end() ? nullptr : it->second;
    });
    LCK(cudaStreamSynchronize(st_));
    return 0;
  }

  int zero() override {
    for (auto& b : bufs_) LCK(cudaMemsetAsync(b.first, 0, b.second * sizeof(R), st_));
    LCK(cudaStreamSynchronize(st_));
    return 0;
  }

  int tl_run(int nsteps, double dt, double t0) override {
    (void)t0;
    if (check_linearisable() || keep_only_state()) return 1;
    if (dt != dt_) drop_graphs(dt);
    for (int s = 0; s < nsteps; ++s) {
      // one captured graph per rotation phase: [TL kernel, forward launch] per launch
      const int ph = m_->phase();
      cudaGraphExec_t& ge = tl_graph_[ph];
      if (!ge) {
        std::vector<Rec> recs;
        if (m_->record_step(dt, &recs)) return fail(m_->error());
        if (capture(&ge, [&] {
              for (const Rec& r : recs) {
                bool done = false;  // the TL launch also did the forward one
                if (tl(r, &done) || (!done && fwd(r))) return 1;
              }
              return 0;
            }))
          return 1;
      }
      LCK(cudaGraphLaunch(ge, st_));
      m_->rotate();
    }
    // pi' ghosts are outputs of nothing: the tangent has none there
    if (L_.nx) zero_ring<R>(D(static_cast<R*>(m_->state_field(4))), L_, st_);
    LCK(cudaStreamSynchronize(st_));
    LCK(cudaGetLastError());
    return 0;
  }

  int ad_run(int nsteps, double dt, double t0, int every) override {
    if (nsteps <= 0) return 0;
    if (check_linearisable()) return 1;
    if (dt != dt_) drop_graphs(dt);
    if (every < 1 && auto_interval(nsteps, dt, &every)) return 1;
    // the undo log for the longest segment, before any segment graph runs
    if (ensure_log(std::min(every, nsteps), dt)) return 1;
    // the adjoint of x_N, uploaded in the slot of the current time-n state;
    // pi' ghosts are no state, so adjoint values there are dropped
    if (L_.nx) zero_ring<R>(D(static_cast<R*>(m_->state_field(4))), L_, st_);
    if (save_lin_state()) return 1;
    // forward pass (the model's own graphs) with segment checkpoints; x_N kept
    // to restore at the end (checkpoint buffers persist across calls)
    const int nseg = (nsteps + every - 1) / every;
    if ((int)snaps_.size() < nseg + 1) snaps_.resize(nseg + 1);
    std::vector<Snap>& segs = snaps_;
    // (the last segment is not run here: its logged replay below is its
    // forward run, and x_N is taken right after it)
    for (int g = 0; g < nseg; ++g) {
      const int s0 = g * every, len = std::min(nsteps, s0 + every) - s0;
      if (snap(&segs[g])) return 1;
      if (g + 1 < nseg && m_->run(len, dt, t0 + s0 * dt)) return fail(m_->error());
    }
    Snap& last = snaps_[nseg];
    // reverse sweep: per segment (last first) one graph replays the segment
    // forward saving every buffer each launch overwrites (the undo log), one
    // graph walks the launches backwards (restore outputs, adjoint kernel);
    // both depend only on the segment's start phase and length
    for (int g = nseg - 1; g >= 0; --g) {
      const int s0 = g * every, len = std::min(nsteps, s0 + every) - s0;
      if (restore(segs[g])) return 1;
      SegGraphs* sg = nullptr;
      if (segment_graphs(segs[g].phase, len, dt, &sg)) return 1;
      LCK(cudaGraphLaunch(sg->fwd, st_));
      if (g == nseg - 1) {
        // the replay ends at x_N, one rotation phase per step further on:
        // keep x_N, and put the adjoint of x_N in the slot of its time-n state
        for (int q = 0; q < len; ++q) m_->rotate();
        if (snap(&last) || zero() || load_lin_state()) return 1;
        for (int q = 0; q < len; ++q) m_->rotate(), m_->rotate();
      }
      LCK(cudaGraphLaunch(sg->rev, st_));
    }
    // dJ/dx0 sits in the slot of x0; move it to the slot of x_N
    if (save_lin_state()) return 1;
    if (restore(last) || zero() || load_lin_state()) return 1;
    LCK(cudaStreamSynchronize(st_));
    LCK(cudaGetLastError());
    return 0;
  }

 private:
  struct Snap {
    int phase = -1;
    R* d = nullptr;  // 8 fields of the time-n state
  };

  R* D(const R* p) const {
    if (!p) return nullptr;
    auto it = map_.find(p);
    return it == map_.end() ? nullptr : static_cast<R*>(it->second);
  }

  template <class A>
  static const A& as(const Rec& r) {
    return *reinterpret_cast<const A*>(r.args.data());
  }

  FillArgs<R> tr(const FillArgs<R>& a) const {
    FillArgs<R> d = a;
    for (int q = 0; q < a.job.n; ++q) d.job.f[q] = D(a.job.f[q]);
    return d;
  }
  FluxArgs<R> tr(const FluxArgs<R>& a) const {
    FluxArgs<R> d = a;
    d.u = D(a.u);
    d.v = D(a.v);
    d.w = D(a.w);
    d.mfx = D(a.mfx);
    d.mfy = D(a.mfy);
    d.mfz = D(a.mfz);
    return d;
  }
  TendArgs<R> tr(const TendArgs<R>& a) const {
    TendArgs<R> d = a;
    for (const R** p : {&d.u, &d.v, &d.w, &d.thp, &d.pip, &d.qv, &d.qc, &d.qr, &d.mfx, &d.mfy,
                        &d.mfz})
      *p = D(*p);
    for (R** p : {&d.tu, &d.tv, &d.tw, &d.tth, &d.tpi, &d.tqv, &d.tqc, &d.tqr, &d.qo_v, &d.qo_c,
                  &d.qo_r})
      *p = D(*p);
    for (const R** p : {&d.qn_v, &d.qn_c, &d.qn_r}) *p = D(*p);
    return d;
  }
  KesArgs<R> tr(const KesArgs<R>& a) const {
    KesArgs<R> d = a;
    for (R** p : {&d.thp, &d.qv, &d.qc, &d.qr}) *p = D(*p);
    d.pip = D(a.pip);
    d.rain = nullptr;  // a diagnostic, not linearised
    return d;
  }
  AcouArgs<R> tr(const AcouArgs<R>& a) const {
    AcouArgs<R> d = a;
    for (const R** p : {&d.u_in, &d.v_in, &d.w_in, &d.pi_prev, &d.pi_cur, &d.th_in, &d.n_pip,
                        &d.n_thp, &d.qv, &d.qc, &d.qr, &d.tu, &d.tv, &d.tw, &d.tth, &d.tpi})
      *p = D(*p);
    for (R** p : {&d.u_out, &d.v_out, &d.w_out, &d.pi_next, &d.th_out}) *p = D(*p);
    return d;
  }

  int unsupported(int kind) { return fail("launch kind " + std::to_string(kind) + " is not linearised"); }

  // replay: a recomputation inside the adjoint sweep, whose rain goes to scratch
  int fwd(const Rec& r, bool replay = false) {
    switch (r.kind) {
      case K_FILL: {
        const auto& a = as<FillArgs<R>>(r);
        launch_fill_ghosts<R>(a.L, a.job, a.open_x, a.open_y, st_);
        break;
      }
      case K_FLUX: {
        const auto& a = as<FluxArgs<R>>(r);
        launch_mass_flux<R>(a.L, a.b, a.m, a.u, a.v, a.w, a.mfx, a.mfy, a.mfz, st_);
        break;
      }
      case K_TEND: launch_tendencies<R>(as<TendArgs<R>>(r), 0, st_); break;
      // the forward u, v and column launches through the variants the model
      // runs (the column adjoint reads the solution from the launch's
      // outputs, whichever kernel wrote them)
      case K_UV:
        if (m_->replay_uv(&as<AcouArgs<R>>(r))) return fail("u, v launch: " + m_->error());
        break;
      case K_COL:
        if (m_->replay_column(&as<AcouArgs<R>>(r))) return fail("acoustic column launch: " + m_->error());
        break;
      case K_KES: {
        KesArgs<R> a = as<KesArgs<R>>(r);
        if (replay) a.rain = rain_scratch_;
        if (launch_kessler<R>(a, st_)) return fail("Kessler launch");
        break;
      }
      default: return unsupported(r.kind);
    }
    return 0;
  }

  int tl(const Rec& r, bool* did_forward) {
    *did_forward = false;
    switch (r.kind) {
      case K_FILL: {
        const FillArgs<R> d = tr(as<FillArgs<R>>(r));
        launch_fill_ghosts<R>(d.L, d.job, d.open_x, d.open_y, st_);
        break;
      }
      case K_FLUX: {
        const FluxArgs<R> d = tr(as<FluxArgs<R>>(r));
        launch_mass_flux<R>(d.L, d.b, d.m, d.u, d.v, d.w, d.mfx, d.mfy, d.mfz, st_);
        break;
      }
      case K_TEND: {
        const auto& a = as<TendArgs<R>>(r);
        tl_tend<R>(a, tr(a), st_);
        break;
      }
      case K_UV: {
        const auto& a = as<AcouArgs<R>>(r);
        tl_uv<R>(a, tr(a), st_);
        break;
      }
      case K_COL: {
        const auto& a = as<AcouArgs<R>>(r);
        if (tl_column<R>(a, tr(a), true, st_)) return fail("column deeper than the linearised kernels hold");
        *did_forward = true;
        break;
      }
      case K_KES: {
        const auto& a = as<KesArgs<R>>(r);
        tl_kessler<R>(a, tr(a), st_);
        break;
      }
      default: return unsupported(r.kind);
    }
    return 0;
  }

  int ad(const Rec& r) {
    switch (r.kind) {
      case K_FILL: ad_fill<R>(tr(as<FillArgs<R>>(r)), st_); break;
      case K_FLUX: ad_flux<R>(tr(as<FluxArgs<R>>(r)), st_); break;
      case K_TEND: {
        const auto& a = as<TendArgs<R>>(r);
        ad_tend<R>(a, tr(a), st_);
        break;
      }
      case K_UV: {
        const auto& a = as<AcouArgs<R>>(r);
        ad_uv<R>(a, tr(a), scr_, st_);
        break;
      }
      case K_COL: {
        const auto& a = as<AcouArgs<R>>(r);
        if (ad_column<R>(a, tr(a), scr_, st_)) return fail("column deeper than the linearised kernels hold");
        break;
      }
      case K_KES: {
        const auto& a = as<KesArgs<R>>(r);
        ad_kessler<R>(a, tr(a), st_);
        break;
      }
      default: return unsupported(r.kind);
    }
    return 0;
  }

  // The adjoint of a column launch while its outputs (w_out, pi_next,
  // th_out: undo-log slots base, base + 1, base + 2) still hold the forward
  // values: w and theta' it updated in place are read from their undo-log
  // copies, the forward solution from w_out and pi_next (no recomputation).
  int ad_column_from_outputs(const Rec& r, size_t base) {
    const auto& a = as<AcouArgs<R>>(r);
    AcouArgs<R> in = a;
    if (a.w_in == a.w_out) in.w_in = log_ + base * n3_;
    if (a.th_in == a.th_out) in.th_in = log_ + (base + 2) * n3_;
    if (ad_column_stored<R>(in, tr(a), scr_, st_)) return fail("column deeper than the linearised kernels hold");
    return 0;
  }

  // forward buffers a launch overwrites (saved before it runs)
  static void outputs(const Rec& r, std::vector<R*>* o) {
    o->clear();
    switch (r.kind) {
      case K_FILL: {
        const auto& a = as<FillArgs<R>>(r);
        for (int q = 0; q < a.job.n; ++q) o->push_back(a.job.f[q]);
        break;
      }
      case K_FLUX: {
        const auto& a = as<FluxArgs<R>>(r);
        *o = {a.mfx, a.mfy, a.mfz};
        break;
      }
      case K_TEND: {
        const auto& a = as<TendArgs<R>>(r);
        *o = {a.tu, a.tv, a.tw, a.tth};
        if (a.tpi) o->push_back(a.tpi);
        if (a.p.moisture) {
          const bool stage = a.qo_v != nullptr;
          o->push_back(stage ? a.qo_v : a.tqv);
          o->push_back(stage ? a.qo_c : a.tqc);
          o->push_back(stage ? a.qo_r : a.tqr);
        }
        break;
      }
      case K_UV: {
        const auto& a = as<AcouArgs<R>>(r);
        *o = {a.u_out, a.v_out};
        break;
      }
      case K_COL: {
        const auto& a = as<AcouArgs<R>>(r);
        *o = {a.w_out, a.pi_next, a.th_out};
        break;
      }
      case K_KES: {
        const auto& a = as<KesArgs<R>>(r);
        *o = {a.thp, a.qv, a.qc, a.qr};
        break;
      }
      default: break;
    }
  }

  // the layout of the case, taken from the first recorded fill
  void learn_layout(const std::vector<Rec>& recs) {
    if (L_.nx) return;
    for (const Rec& r : recs)
      if (r.kind == K_FILL) {
        L_ = as<FillArgs<R>>(r).L;
        return;
      }
  }

  struct SegGraphs {
    cudaGraphExec_t fwd = nullptr, rev = nullptr;
  };

  template <class F>
  int capture(cudaGraphExec_t* out, F&& issue) {
    cudaGraph_t gr = nullptr;
    LCK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
    const int rc = issue();
    cudaError_t ce = cudaStreamEndCapture(st_, &gr);
    if (rc) {
      if (gr) cudaGraphDestroy(gr);
      return 1;
    }
    if (ce != cudaSuccess) return fail(std::string("graph capture: ") + cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(out, gr, 0);
    cudaGraphDestroy(gr);
    if (ie != cudaSuccess) return fail(std::string("graph instantiate: ") + cudaGetErrorString(ie));
    return 0;
  }

  void drop_graphs(double dt) {
    for (auto& ge : tl_graph_)
      if (ge) {
        cudaGraphExecDestroy(ge);
        ge = nullptr;
      }
    drop_segment_graphs();
    dt_ = dt;
  }

  void drop_segment_graphs() {
    for (auto& kv : seg_) {
      if (kv.second.fwd) cudaGraphExecDestroy(kv.second.fwd);
      if (kv.second.rev) cudaGraphExecDestroy(kv.second.rev);
    }
    seg_.clear();
  }

  // undo-log slots (whole fields) one step needs: the outputs of its launches
  int slots_per_step(double dt, size_t* out) {
    std::vector<std::vector<Rec>> recs;
    if (record_segment(m_->phase(), 1, dt, &recs)) return 1;
    size_t slots = 0;
    std::vector<R*> o;
    for (const Rec& r : recs[0]) {
      outputs(r, &o);
      slots += o.size();
    }
    *out = slots;
    return 0;
  }

  // An undo log for segments of up to `len` steps.  The segment graphs hold
  // the log's address, so a new log first retires every one of them (after
  // the stream has drained): none may run on a freed log.
  int ensure_log(int len, double dt) {
    size_t per = 0;
    if (slots_per_step(dt, &per)) return 1;
    const size_t slots = per * (size_t)len;
    if (slots <= log_cap_) return 0;
    LCK(cudaStreamSynchronize(st_));
    drop_segment_graphs();
    if (log_) cudaFree(log_);
    log_ = nullptr;
    log_cap_ = 0;
    LCK(cudaMalloc(&log_, slots * n3_ * sizeof(R)));
    log_cap_ = slots;
    return 0;
  }

  // the launches of `len` steps from rotation phase `phase` (the model is
  // left at its current phase)
  int record_segment(int phase, int len, double dt, std::vector<std::vector<Rec>>* recs) {
    const int keep = m_->phase();
    while (m_->phase() != phase) m_->rotate();
    recs->assign(len, {});
    for (int s = 0; s < len; ++s) {
      if (m_->record_step(dt, &(*recs)[s])) return fail(m_->error());
      m_->rotate();
    }
    while (m_->phase() != keep) m_->rotate();
    return 0;
  }

  // The longest checkpoint interval whose undo log fits in 80 % of the free
  // device memory (plus the log already held): with one segment the sweep
  // recomputes nothing (the logged replay is the only forward run).
  int auto_interval(int nsteps, double dt, int* every) {
    size_t slots = 0;
    if (slots_per_step(dt, &slots)) return 1;
    size_t free_b = 0, total_b = 0;
    LCK(cudaMemGetInfo(&free_b, &total_b));
    const double per_step = (double)slots * n3_ * sizeof(R);
    const double room = 0.8 * (double)free_b + (double)log_cap_ * n3_ * sizeof(R);
    long n = per_step > 0 ? (long)(room / per_step) : nsteps;
    if (n > nsteps) n = nsteps;
    *every = n < 1 ? 1 : (int)n;
    return 0;
  }

  int segment_graphs(int phase, int len, double dt, SegGraphs** out) {
    const long key = (long)phase * 1000000L + len;
    auto it = seg_.find(key);
    if (it != seg_.end()) {
      *out = &it->second;
      return 0;
    }
    std::vector<std::vector<Rec>> recs;
    if (record_segment(phase, len, dt, &recs)) return 1;
    size_t slots = 0;
    std::vector<R*> o;
    for (auto& st : recs)
      for (const Rec& r : st) {
        outputs(r, &o);
        slots += o.size();
      }
    if (!rain_scratch_) LCK(cudaMalloc(&rain_scratch_, L_.n2() * sizeof(R)));
    if (slots > log_cap_) return fail("undo log smaller than the segment (ensure_log not called)");
    SegGraphs g;
    if (capture(&g.fwd, [&] {
          size_t slot = 0;
          std::vector<R*> oo;
          for (auto& st : recs)
            for (const Rec& r : st) {
              outputs(r, &oo);
              CopyJob<R> job{};
              for (R* p : oo) {
                job.src[job.count] = p;
                job.dst[job.count++] = log_ + slot * n3_;
                ++slot;
              }
              if (copy_fields<R>(job, n3_, st_)) return fail("undo-log copy");
              if (fwd(r, true)) return 1;
            }
          return 0;
        }))
      return 1;
    if (capture(&g.rev, [&] {
          size_t slot = slots;
          std::vector<R*> oo;
          for (size_t s = recs.size(); s-- > 0;)
            for (size_t q = recs[s].size(); q-- > 0;) {
              const Rec& r = recs[s][q];
              outputs(r, &oo);
              // a column launch's adjoint runs before its outputs are
              // restored: it reads the forward solution from them
              const bool col = r.kind == K_COL;
              if (col && ad_column_from_outputs(r, slot - oo.size())) return 1;
              CopyJob<R> job{};
              for (size_t z = oo.size(); z-- > 0;) {
                --slot;
                job.src[job.count] = log_ + slot * n3_;
                job.dst[job.count++] = oo[z];
              }
              if (copy_fields<R>(job, n3_, st_)) return fail("undo-log copy");
              if (!col && ad(r)) return 1;
            }
          return 0;
        }))
      return 1;
    *out = &(seg_[key] = g);
    return 0;
  }

  int snap(Snap* s) {
    if (!s->d) LCK(cudaMalloc(&s->d, 8 * n3_ * sizeof(R)));
    s->phase = m_->phase();
    for (int f = 0; f < 8; ++f)
      LCK(cudaMemcpyAsync(s->d + f * n3_, m_->state_field(f), n3_ * sizeof(R),
                          cudaMemcpyDeviceToDevice, st_));
    return 0;
  }

  int restore(const Snap& s) {
    if (s.phase < 0 || s.phase > 2 || !s.d) return fail("restore of a state never saved");
    while (m_->phase() != s.phase) m_->rotate();
    for (int f = 0; f < 8; ++f)
      LCK(cudaMemcpyAsync(m_->state_field(f), s.d + f * n3_, n3_ * sizeof(R),
                          cudaMemcpyDeviceToDevice, st_));
    return 0;
  }

  void free_snap(Snap* s) {
    if (s->d) cudaFree(s->d);
    s->d = nullptr;
  }

  // a copy of the linearised time-n state (8 fields) in a buffer kept for
  // the context's lifetime
  int save_lin_state() {
    if (!hold_) LCK(cudaMalloc(&hold_, 8 * n3_ * sizeof(R)));
    for (int f = 0; f < 8; ++f)
      LCK(cudaMemcpyAsync(hold_ + f * n3_, D(static_cast<R*>(m_->state_field(f))), n3_ * sizeof(R),
                          cudaMemcpyDeviceToDevice, st_));
    return 0;
  }

  int load_lin_state() {
    for (int f = 0; f < 8; ++f)
      LCK(cudaMemcpyAsync(D(static_cast<R*>(m_->state_field(f))), hold_ + f * n3_, n3_ * sizeof(R),
                          cudaMemcpyDeviceToDevice, st_));
    return 0;
  }

  // zero every linearised buffer but the time-n state's
  int keep_only_state() {
    if (save_lin_state() || zero() || load_lin_state()) return 1;
    LCK(cudaStreamSynchronize(st_));
    return 0;
  }

  int fail(const std::string& m) {
    err_ = m;
    return 1;
  }

  // switches turned on after wfe_lin_enable (a boundary relaxation, surface
  // physics) make the recorded step one the kernels do not linearise
  int check_linearisable() {
    std::string why;
    return m_->linearisable(&why) ? 0 : fail(why);
  }

  void release() {
    drop_graphs(0);
    if (m_) m_->set_lin_map(nullptr);
    for (auto& b : bufs_) cudaFree(b.first);
    bufs_.clear();
    if (log_) cudaFree(log_);
    log_ = nullptr;
    if (rain_scratch_) cudaFree(rain_scratch_);
    rain_scratch_ = nullptr;
    for (R*& f : scr_.f) {
      if (f) cudaFree(f);
      f = nullptr;
    }
    for (auto& sn : snaps_) free_snap(&sn);
    snaps_.clear();
    if (hold_) cudaFree(hold_);
    hold_ = nullptr;
  }

  Model* m_ = nullptr;
  cudaStream_t st_ = nullptr;
  std::map<const void*, void*> map_;
  std::vector<std::pair<R*, size_t>> bufs_, fwd_;
  size_t n3_ = 0;
  Layout L_{};
  R* log_ = nullptr;
  size_t log_cap_ = 0;
  R* rain_scratch_ = nullptr;  // rain of the adjoint sweep's forward replays
  LinScratch<R> scr_{};        // work fields of the gather-form adjoints
  std::vector<Snap> snaps_;    // adjoint checkpoints, kept across calls
  R* hold_ = nullptr;          // a saved linearised time-n state
  double dt_ = -1;
  cudaGraphExec_t tl_graph_[3] = {nullptr, nullptr, nullptr};
  std::map<long, SegGraphs> seg_;
};

}  // namespace

Lin* Lin::create(Model* m, std::string* err) {
  if (!m) {
    *err = "no model";
    return nullptr;
  }
  Lin* l = nullptr;
  int rc;
  if (m->fp64()) {
    auto* t = new LinT<double>();
    rc = t->init(m);
    l = t;
  } else {
    auto* t = new LinT<float>();
    rc = t->init(m);
    l = t;
  }
  if (rc) {
    *err = l->error();
    delete l;
    return nullptr;
  }
  return l;
}

}  // namespace wfe
