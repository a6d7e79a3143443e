// serve.cpp -- many FEL runs on one GPU: the batched parameter scan and the
// served request stream, both on the g4b_batch engine.
//
// A job is one mixed-precision run (its own slice count, grid, particle
// count, taper, detuning, seed power and length) on a shared lattice.  Host
// inputs (quiet-start beam, Gaussian seed, per-step tables) are prepared by
// worker threads; device state lives in a g4b_run attached to the batch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "g4h.h"
#include "g4h_internal.h"
#include "genesis4.h"

namespace g4h {

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Host inputs of one job, ready to upload.
struct JobInputs {
  int index = -1;
  std::vector<int64_t> off;
  std::vector<double> x, y, px, py, g, th, cells, current;
  std::vector<g4b_step> steps;
  std::vector<double> fc, slip;
  double dgrid = 0, ks = 0;
};

bool prepare(const g4h_engine_config& cfg, const Undulator& lat, const g4h_job& j, int index,
             JobInputs& in) {
  in.index = index;
  const int ns = j.nslice, n = j.ngrid;
  const size_t np = (size_t)ns * j.npart;
  g4h_beam_spec sp{};
  sp.nslice = ns;
  sp.npart = j.npart;
  sp.nbins = 4;
  sp.shotnoise = j.shotnoise;
  sp.seed = j.seed;
  sp.gamma0 = j.gamma;
  sp.delgam = j.delgam;
  sp.ex = sp.ey = j.emit;
  sp.betax = sp.betay = j.beta;
  sp.reflength = cfg.lambda0;
  sp.slicelength = cfg.lambda0;
  in.current.assign(ns, j.current);
  in.off.resize(ns + 1);
  for (auto* v : {&in.x, &in.y, &in.px, &in.py, &in.g, &in.th}) v->resize(np);
  if (g4h_load_beam(&sp, in.current.data(), in.x.data(), in.y.data(), in.px.data(),
                    in.py.data(), in.g.data(), in.th.data(), in.off.data()) != G4B_OK)
    return false;
  std::vector<double> plane(2 * (size_t)n * n);
  if (g4h_gaussian_field(n, j.gridmax, cfg.lambda0, j.seed_power, j.waist, plane.data()) !=
      G4B_OK)
    return false;
  in.cells.resize(plane.size() * ns);
  for (int s = 0; s < ns; ++s)
    std::memcpy(in.cells.data() + plane.size() * s, plane.data(), plane.size() * 8);
  const int nst = std::min(j.nsteps, lat.nstep());
  in.steps.resize(nst);
  in.fc.resize(nst);
  in.slip.resize(nst);
  const double zend = lat.steps[nst - 1].z;
  for (int i = 0; i < nst; ++i) {
    LatticeStep ls = lat.steps[i];
    if (ls.st.in_undulator) {  // linear taper d(aw)/aw over the run
      const double zm = ls.z - 0.5 * ls.st.delz;
      ls.st.aw *= 1.0 - j.taper * zm / zend;
    }
    in.steps[i] = ls.st;
    in.fc[i] = ls.st.in_undulator ? coupling(ls.st.aw, 1, ls.helical != 0) : 0.0;
    in.slip[i] = ls.slip;
  }
  in.dgrid = 2 * j.gridmax / (n - 1);
  in.ks = 2 * M_PI / cfg.lambda0;
  return true;
}

// Device bytes a job will hold (particles 28 B, per plane a + b + source tile,
// diagnostics history of one step), for admission.
double estimate_bytes(const g4h_job& j) {
  const double n = j.ngrid, ld = n + ((int)n & 1);
  const double planes = 3.0 * j.nslice * n * ld * 8;
  return 28.0 * j.nslice * j.npart + planes + 4096.0 * j.nslice + (1 << 20);
}

int create_run(g4b_ctx* ctx, const g4h_engine_config& cfg, const g4h_job& j,
               const JobInputs& in, g4b_run** out) {
  g4b_run_desc d{};
  d.nslice = j.nslice;
  d.nfield = 1;
  d.harm[0] = 1;
  d.ngrid[0] = j.ngrid;
  d.gridmax[0] = j.gridmax;
  d.lambda0 = cfg.lambda0;
  d.gamma_ref = cfg.gamma_ref;
  d.sample = 1.0;
  d.time_run = j.time_run;
  d.periodic = 0;
  d.nbunch = 1;
  d.precision = G4B_MIXED;
  g4b_run* r = nullptr;
  int rc = g4b_run_create(ctx, &d, in.off.data(), &r);
  if (rc) return rc;
  const int nst = (int)in.steps.size();
  if ((rc = g4b_run_upload_beam(r, in.x.data(), in.y.data(), in.px.data(), in.py.data(),
                                in.g.data(), in.th.data())) ||
      (rc = g4b_run_upload_field(r, 0, in.cells.data(), 0)) ||
      (rc = g4b_run_set_current(r, in.current.data())) ||
      (rc = g4b_run_set_lattice(r, nst, in.steps.data(), in.fc.data(), in.slip.data(), 1))) {
    g4b_run_destroy(r);
    return rc;
  }
  *out = r;
  return G4B_OK;
}

// Final output of a finished job: total power [W] of its last step and the
// raw diagnostic records of that step (beam [nslice][25], field [nslice][9]).
void collect(g4b_run* r, const g4h_job& j, const JobInputs& in, double* power,
             std::vector<double>& rec) {
  const int ns = j.nslice;
  std::vector<double> hb((size_t)ns * 25), hf((size_t)ns * 9);
  g4b_run_history(r, (int)in.steps.size() - 1, hb.data(), hf.data());
  const double scl = in.dgrid * eev / in.ks;
  double p = 0;
  for (int s = 0; s < ns; ++s) p += hf[(size_t)s * 9] * scl * scl / vacimp;
  *power = p;
  rec = hb;
  rec.insert(rec.end(), hf.begin(), hf.end());
}

// Worker pool preparing job inputs in index order into a bounded queue.
class Producer {
 public:
  Producer(const g4h_engine_config& cfg, const Undulator& lat, const g4h_job* jobs, int njobs,
           int threads, int depth)
      : cfg_(cfg), lat_(lat), jobs_(jobs), njobs_(njobs), depth_(depth) {
    for (int t = 0; t < std::max(1, threads); ++t) pool_.emplace_back([this] { work(); });
  }
  ~Producer() {
    {
      std::lock_guard<std::mutex> l(m_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : pool_) t.join();
  }
  // Inputs of job `i` if ready (nullptr otherwise); the caller takes them.
  std::unique_ptr<JobInputs> take(int i, bool wait) {
    std::unique_lock<std::mutex> l(m_);
    for (;;) {
      for (auto it = ready_.begin(); it != ready_.end(); ++it)
        if ((*it)->index == i) {
          auto p = std::move(*it);
          ready_.erase(it);
          cv_.notify_all();
          return p;
        }
      if (!wait || failed_) return nullptr;
      cv_.wait(l);
    }
  }
  bool failed() const { return failed_; }

 private:
  void work() {
    for (;;) {
      int i;
      {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return stop_ || (next_ < njobs_ && inflight_ + (int)ready_.size() < depth_); });
        if (stop_) return;
        i = next_++;
        ++inflight_;
      }
      auto in = std::make_unique<JobInputs>();
      const bool ok = prepare(cfg_, lat_, jobs_[i], i, *in);
      {
        std::lock_guard<std::mutex> l(m_);
        --inflight_;
        if (!ok) failed_ = true;
        else ready_.push_back(std::move(in));
      }
      cv_.notify_all();
    }
  }
  const g4h_engine_config& cfg_;
  const Undulator& lat_;
  const g4h_job* jobs_;
  int njobs_, depth_;
  std::mutex m_;
  std::condition_variable cv_;
  std::vector<std::thread> pool_;
  std::deque<std::unique_ptr<JobInputs>> ready_;
  int next_ = 0, inflight_ = 0;
  bool stop_ = false;
  std::atomic<bool> failed_{false};
};

int build_shared_lattice(const g4h_engine_config* cfg, Undulator& lat) {
  if (!cfg || !cfg->lattice || !cfg->beamline) {
    set_error("engine: lattice and beamline required");
    return G4B_ERR_ARG;
  }
  if (!build_lattice(cfg->lattice, cfg->beamline, cfg->delz, cfg->gamma_ref, cfg->lambda0, lat))
    return G4B_ERR_ARG;
  return G4B_OK;
}

int threads_for(const g4h_engine_config* cfg) {
  if (cfg->threads > 0) return cfg->threads;
  const unsigned h = std::thread::hardware_concurrency();
  return h > 2 ? (int)h - 2 : 1;
}

}  // namespace

}  // namespace g4h

using namespace g4h;

extern "C" {

// Batched scan: every job resident at once, advanced together (mode 0) or one
// after another through the single-run graph path (mode 1).  Host input
// preparation and uploads are outside the timed loop.
int g4h_scan(const g4h_engine_config* cfg, const g4h_job* jobs, int njobs,
             g4h_scan_result* res, double* final_power, double* records) {
  if (!cfg || !jobs || njobs < 1 || !res) {
    set_error("g4h_scan: bad argument");
    return G4B_ERR_ARG;
  }
  try {
    Undulator lat;
    if (int rc = build_shared_lattice(cfg, lat)) return rc;
    g4b_ctx* ctx = cuda_context();
    std::vector<std::unique_ptr<JobInputs>> ins(njobs);
    {
      Producer prod(*cfg, lat, jobs, njobs, threads_for(cfg), njobs);
      for (int i = 0; i < njobs; ++i) {
        ins[i] = prod.take(i, true);
        if (!ins[i]) {
          set_error("g4h_scan: input preparation failed");
          return G4B_ERR_ARG;
        }
      }
    }
    std::vector<g4b_run*> runs(njobs, nullptr);
    auto cleanup = [&] {
      for (auto* r : runs)
        if (r) g4b_run_destroy(r);
    };
    for (int i = 0; i < njobs; ++i)
      if (int rc = create_run(ctx, *cfg, jobs[i], *ins[i], &runs[i])) {
        cleanup();
        return rc;
      }
    int maxst = 0;
    double slice_steps = 0;
    for (int i = 0; i < njobs; ++i) {
      const int nst = (int)ins[i]->steps.size();
      maxst = std::max(maxst, nst);
      slice_steps += (double)jobs[i].nslice * nst;
    }
    g4b_batch* batch = nullptr;
    if (cfg->mode == 0) {
      if (int rc = g4b_batch_create(ctx, njobs, &batch)) {
        cleanup();
        return rc;
      }
      for (int i = 0; i < njobs; ++i) {
        int slot;
        g4b_batch_attach(batch, runs[i], 0, (int)ins[i]->steps.size(), &slot);
      }
      // the tuner times its candidate shapes on the first steps of the
      // real runs (launch shapes do not change results; with tune = 2 it
      // also picks the ADI row layouts, which set the FP32 rounding)
      if (cfg->tune >= 2)
        g4b_batch_tune_layouts(batch);
      else if (cfg->tune)
        g4b_batch_tune(batch);
    }
    check(g4b_ctx_synchronize(ctx), "g4h_scan");
    const double t0 = now_s();
    if (cfg->mode == 0) {
      check(g4b_batch_step(batch, maxst, cfg->use_graph), "g4h_scan");
    } else {
      for (int i = 0; i < njobs; ++i)
        check(g4b_run_advance(runs[i], 0, (int)ins[i]->steps.size(), cfg->use_graph),
              "g4h_scan");
    }
    check(g4b_ctx_synchronize(ctx), "g4h_scan");
    const double t1 = now_s();
    res->seconds = t1 - t0;
    res->slice_steps = slice_steps;
    res->value = slice_steps / res->seconds;
    res->njobs = njobs;
    res->grids[0] = res->grids[1] = res->grids[2] = res->grids[3] = 0;
    if (batch) g4b_batch_shapes(batch, res->grids);
    res->layouts_16 = res->layouts_switched = 0;
    for (int i = 0; i < njobs; ++i) {
      int modes[8] = {0};
      g4b_run_get_layouts(runs[i], modes);
      res->layouts_16 += modes[0] >= 100;
      res->layouts_switched += modes[0] != g4b_default_layout(jobs[i].ngrid);
    }
    uint64_t bytes = 0;
    for (auto* r : runs) {
      uint64_t b = 0;
      g4b_run_device_bytes(r, &b);
      bytes += b;
    }
    res->device_bytes = (double)bytes;
    size_t roff = 0;
    for (int i = 0; i < njobs; ++i) {
      double p;
      std::vector<double> rec;
      collect(runs[i], jobs[i], *ins[i], &p, rec);
      if (final_power) final_power[i] = p;
      if (records) {
        std::memcpy(records + roff, rec.data(), rec.size() * 8);
        roff += rec.size();
      }
    }
    if (batch) g4b_batch_destroy(batch);
    cleanup();
    return G4B_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return G4B_ERR_CUDA;
  }
}

// Served request stream with continuous batching.  Request i arrives at
// arrival[i] seconds after the start.  Admission threads (each with its own
// context and stream) prepare a request's inputs ahead of time; once it has
// arrived, a batch slot is free and the free device memory minus the reserve
// covers its estimated footprint, they create and upload its device state.
// The step loop attaches admitted requests between steps, advances every
// admitted request by one lattice step per batch step (one step kept in
// flight), and when a request's last step has completed on the device reads
// its final diagnostics back and frees it.  latency[i] = completion - arrival.
int g4h_serve(const g4h_engine_config* cfg, const g4h_job* jobs, const double* arrival,
              int njobs, double* latency, double* final_power, double* records,
              g4h_serve_stats* stats) {
  if (!cfg || !jobs || !arrival || njobs < 1 || !latency || !stats) {
    set_error("g4h_serve: bad argument");
    return G4B_ERR_ARG;
  }
  try {
    Undulator lat;
    if (int rc = build_shared_lattice(cfg, lat)) return rc;
    g4b_ctx* ctx = cuda_context();
    const int max_runs = std::max(1, cfg->max_runs);
    g4b_batch* batch = nullptr;
    if (int rc = g4b_batch_create(ctx, max_runs, &batch)) return rc;
    struct Ready {
      int job;
      g4b_run* run;
      std::unique_ptr<JobInputs> in;
    };
    std::mutex m;
    std::condition_variable cv;
    std::deque<Ready> ready;
    int claimed = 0, slots_used = 0;
    double reserved = 0;  // bytes promised to requests being created
    bool stop = false, failed = false;
    std::string err;
    const double t0 = now_s();
    auto worker = [&]() {
     try {
      g4b_ctx* wc = nullptr;
      if (g4b_ctx_create(0, &wc) != G4B_OK) {
        std::lock_guard<std::mutex> l(m);
        failed = true;
        err = g4b_last_error();
        cv.notify_all();
        return;
      }
      for (;;) {
        int i;
        {
          std::unique_lock<std::mutex> l(m);
          if (stop || failed || claimed >= njobs) break;
          i = claimed++;
        }
        auto in = std::make_unique<JobInputs>();
        if (!prepare(*cfg, lat, jobs[i], i, *in)) {
          std::lock_guard<std::mutex> l(m);
          failed = true;
          err = "input preparation failed";
          cv.notify_all();
          break;
        }
        // wait for the arrival, then for a slot and memory
        const double wait = arrival[i] - (now_s() - t0);
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
        const double need = estimate_bytes(jobs[i]);
        {
          std::unique_lock<std::mutex> l(m);
          for (;;) {
            if (stop || failed) break;
            if (slots_used < max_runs) {
              uint64_t fb = 0, tb = 0;
              g4b_ctx_mem_info(wc, &fb, &tb);
              if ((double)fb - reserved - cfg->reserve_bytes >= need) break;
            }
            cv.wait_for(l, std::chrono::milliseconds(1));
          }
          if (stop || failed) break;
          ++slots_used;
          reserved += need;
        }
        g4b_run* r = nullptr;
        const int rc = create_run(wc, *cfg, jobs[i], *in, &r);
        std::lock_guard<std::mutex> l(m);
        reserved -= need;
        if (rc != G4B_OK) {
          failed = true;
          err = g4b_last_error();
          --slots_used;
          cv.notify_all();
          break;
        }
        ready.push_back(Ready{i, r, std::move(in)});
        cv.notify_all();
      }
      g4b_ctx_destroy(wc);  // released once its runs are destroyed
     } catch (const std::exception& e) {
      std::lock_guard<std::mutex> l(m);
      failed = true;
      err = e.what();
      cv.notify_all();
     }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads_for(cfg); ++t) pool.emplace_back(worker);
    struct Active {
      int job = -1, slot = -1;
      g4b_run* run = nullptr;
      std::unique_ptr<JobInputs> in;
      uint64_t done_ticket = 0;  // mark after the last step, + 1 (0 = none yet)
      bool last_launched = false;
    };
    std::vector<Active> act;
    std::vector<size_t> rec_off(njobs + 1, 0);
    for (int i = 0; i < njobs; ++i) rec_off[i + 1] = rec_off[i] + (size_t)jobs[i].nslice * 34;
    int finished = 0, peak = 0;
    double slice_steps = 0, batch_steps = 0;
    uint64_t last_ticket = 0;
    bool have_ticket = false;
    int rc_loop = G4B_OK;
    try {
    while (finished < njobs) {
      {  // attach admitted requests
        std::unique_lock<std::mutex> l(m);
        if (failed) {
          set_error("g4h_serve: " + err);
          rc_loop = G4B_ERR_CUDA;
          break;
        }
        if (act.empty() && ready.empty())
          cv.wait_for(l, std::chrono::milliseconds(1));
        while (!ready.empty()) {
          Ready rd = std::move(ready.front());
          ready.pop_front();
          Active a;
          a.job = rd.job;
          a.run = rd.run;
          a.in = std::move(rd.in);
          const int nst = (int)a.in->steps.size();
          if (g4b_batch_attach(batch, a.run, 0, nst, &a.slot) != G4B_OK) {
            rc_loop = G4B_ERR_STATE;
            break;
          }
          act.push_back(std::move(a));
        }
        if (rc_loop) break;
      }
      peak = std::max(peak, (int)act.size());
      int running = 0;
      for (auto& a : act) {
        int nxt = 0, rem = 0;
        g4b_batch_status(batch, a.slot, &nxt, &rem);
        if (rem > 0) {
          ++running;
          slice_steps += jobs[a.job].nslice;
          if (rem == 1) a.last_launched = true;
        }
      }
      if (running > 0) {
        check(g4b_batch_step(batch, 1, cfg->use_graph), "g4h_serve");
        uint64_t tk;
        check(g4b_ctx_mark(ctx, &tk), "g4h_serve");
        for (auto& a : act)
          if (a.last_launched && a.done_ticket == 0) a.done_ticket = tk + 1;
        if (have_ticket) {  // keep one step in flight
          int d;
          check(g4b_ctx_mark_query(ctx, last_ticket, 1, &d), "g4h_serve");
        }
        last_ticket = tk;
        have_ticket = true;
        batch_steps += 1;
      }
      for (size_t k = 0; k < act.size();) {
        Active& a = act[k];
        int done = 0;
        if (a.done_ticket)
          check(g4b_ctx_mark_query(ctx, a.done_ticket - 1, 0, &done), "g4h_serve");
        if (!done) {
          ++k;
          continue;
        }
        latency[a.job] = (now_s() - t0) - arrival[a.job];
        double p;
        std::vector<double> rec;
        collect(a.run, jobs[a.job], *a.in, &p, rec);
        if (final_power) final_power[a.job] = p;
        if (records) std::memcpy(records + rec_off[a.job], rec.data(), rec.size() * 8);
        check(g4b_batch_detach(batch, a.slot), "g4h_serve");
        g4b_run_destroy(a.run);
        act.erase(act.begin() + k);
        ++finished;
        std::lock_guard<std::mutex> l(m);
        --slots_used;
        cv.notify_all();
      }
    }
    } catch (const std::exception& e) {
      set_error(std::string("g4h_serve: ") + e.what());
      rc_loop = G4B_ERR_CUDA;
    }
    {
      std::lock_guard<std::mutex> l(m);
      stop = true;
      cv.notify_all();
    }
    for (auto& t : pool) t.join();
    for (auto& rd : ready) g4b_run_destroy(rd.run);
    for (auto& a : act) g4b_run_destroy(a.run);
    const double t1 = now_s();
    g4b_ctx_synchronize(ctx);
    g4b_batch_destroy(batch);
    if (rc_loop) {
      const std::string msg = g4h::last_error();
      g4h::set_error(msg);
      return rc_loop;
    }
    std::vector<double> l(latency, latency + njobs);
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) {
      const double pos = q * (njobs - 1);
      const int lo = (int)std::floor(pos), hi = std::min(njobs - 1, lo + 1);
      return l[lo] + (l[hi] - l[lo]) * (pos - lo);
    };
    stats->seconds = t1 - t0;
    stats->p50 = pct(0.50);
    stats->p99 = pct(0.99);
    stats->mean = 0;
    for (double v : l) stats->mean += v / njobs;
    stats->requests_per_s = njobs / stats->seconds;
    stats->slice_steps = slice_steps;
    stats->slice_steps_per_s = slice_steps / stats->seconds;
    stats->peak_concurrency = peak;
    stats->batch_steps = batch_steps;
    return G4B_OK;
  } catch (const std::exception& e) {
    set_error(e.what());
    return G4B_ERR_CUDA;
  }
}

}  // extern "C"
