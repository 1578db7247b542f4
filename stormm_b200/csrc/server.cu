// Request server: continuous batching of conformer-minimization requests on one GPU.
//
// Requests arrive on any host thread (sb_server_submit copies the topology and coordinates) and
// wait in a queue.  One worker thread owns the GPU side:
//   admit     while fewer than max_batches batches are in flight, take queued requests in
//             arrival order while the estimated device memory of the molecules in flight stays
//             within the HBM budget, build a synthesis of them on a stream of the batch's own
//             (stream-ordered allocations, so building never waits for other batches), upload
//             coordinates, reset the minimizer and launch the first cycles_per_launch cycles
//   poll      when a batch's launch has finished (event query, no blocking), read every
//             molecule's progress, retire the molecules that converged or reached the cycle cap
//             (final energies and coordinates are copied out), and launch the next cycles for
//             the rest; a batch whose molecules have all retired is freed on its stream
//   migrate   when at most a quarter of a minimization batch is still running and new
//             minimizations wait, the running molecules' minimizer states are read out, they
//             go back to the front of the queue and the batch is freed; admitted again with
//             the waiting requests they continue from their states (slot backfill)
// Batches overlap on the device, new batches start while older ones run (backfill), and a
// molecule's trajectory is bit-identical whichever batch, unit or launch split it gets.
//
// Errors stay with the requests that cause them.  submit runs the synthesis's topology checks on
// the host, so a malformed topology is refused before it is queued.  A batch that still fails
// to build is released and its requests queued again to be admitted one per batch, so that only
// the request that cannot be built fails; a batch whose launch or read-back fails returns its
// unfinished requests with the error code.  Either way the worker goes on with the other
// batches, unless the CUDA context itself is lost.
#include <cuda_runtime.h>

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

#include "stormm_b200.h"
#include "synthesis.h"

namespace sb {

namespace {

template <typename T> void copyArray(std::vector<T>* dst, const T* src, size_t n) {
  if (src != nullptr && n > 0) {
    dst->assign(src, src + n);
  }
  else {
    dst->clear();
  }
}

template <typename T> const T* ptrOrNull(const std::vector<T> &v) {
  return v.empty() ? nullptr : v.data();
}

// A request's own copy of its topology and coordinates
struct Request {
  long long id = 0;
  int natom = 0;
  int n_lj = 0;
  int nbond = 0;
  int nangl = 0;
  int ndihe = 0;
  std::vector<double> charge, lja, ljb, lja14, ljb14, pb_radii, gb_screen, gb_alpha, gb_beta;
  std::vector<double> gb_gamma, bond_keq, bond_leq, angl_keq, angl_theta0, dihe_amp, dihe_freq;
  std::vector<double> dihe_phase, dihe_scee, dihe_scnb, xyz;
  std::vector<int> lj_idx, excl_bounds, excl_list, bond_atoms, angl_atoms, dihe_atoms;
  std::vector<int> dihe_improper;
  int nubrd = 0, ncimp = 0, ncmap = 0, ncmap_surf = 0;
  std::vector<int> ubrd_atoms, cimp_atoms, cmap_atoms, cmap_surface, cmap_dims;
  std::vector<double> ubrd_keq, ubrd_leq, cimp_keq, cimp_phase, cmap_values;
  double bytes = 0.0;
  double t_submit = 0.0;
  double t_admit = 0.0;
  int kind = SB_REQUEST_MINIMIZE;
  bool solo = false;                  // retried alone after its batch failed to build
  // minimizer state carried over from the batch the request ran in before (null: fresh)
  std::shared_ptr<MinimizerState> state;

  Request(const sb_topology &t, const double* coords) {
    natom = t.natom;
    n_lj = t.n_lj_types;
    nbond = t.nbond;
    nangl = t.nangl;
    ndihe = t.ndihe;
    const size_t n = natom;
    const size_t nt2 = static_cast<size_t>(n_lj) * n_lj;
    copyArray(&charge, t.charge, n);
    copyArray(&lj_idx, t.lj_idx, n);
    copyArray(&lja, t.lja, nt2);
    copyArray(&ljb, t.ljb, nt2);
    copyArray(&lja14, t.lja14, nt2);
    copyArray(&ljb14, t.ljb14, nt2);
    copyArray(&excl_bounds, t.excl_bounds, n + 1);
    const size_t nexcl = (t.excl_bounds != nullptr) ? static_cast<size_t>(t.excl_bounds[n]) : 0;
    copyArray(&excl_list, t.excl_list, nexcl);
    copyArray(&pb_radii, t.pb_radii, n);
    copyArray(&gb_screen, t.gb_screen, n);
    copyArray(&gb_alpha, t.gb_alpha, n);
    copyArray(&gb_beta, t.gb_beta, n);
    copyArray(&gb_gamma, t.gb_gamma, n);
    copyArray(&bond_atoms, t.bond_atoms, 2 * static_cast<size_t>(nbond));
    copyArray(&bond_keq, t.bond_keq, nbond);
    copyArray(&bond_leq, t.bond_leq, nbond);
    copyArray(&angl_atoms, t.angl_atoms, 3 * static_cast<size_t>(nangl));
    copyArray(&angl_keq, t.angl_keq, nangl);
    copyArray(&angl_theta0, t.angl_theta0, nangl);
    copyArray(&dihe_atoms, t.dihe_atoms, 4 * static_cast<size_t>(ndihe));
    copyArray(&dihe_amp, t.dihe_amp, ndihe);
    copyArray(&dihe_freq, t.dihe_freq, ndihe);
    copyArray(&dihe_phase, t.dihe_phase, ndihe);
    copyArray(&dihe_scee, t.dihe_scee, ndihe);
    copyArray(&dihe_scnb, t.dihe_scnb, ndihe);
    copyArray(&dihe_improper, t.dihe_improper, ndihe);
    nubrd = t.nubrd;
    ncimp = t.ncimp;
    ncmap = t.ncmap;
    ncmap_surf = (t.ncmap > 0) ? t.ncmap_surf : 0;
    copyArray(&ubrd_atoms, t.ubrd_atoms, 2 * static_cast<size_t>(nubrd));
    copyArray(&ubrd_keq, t.ubrd_keq, nubrd);
    copyArray(&ubrd_leq, t.ubrd_leq, nubrd);
    copyArray(&cimp_atoms, t.cimp_atoms, 4 * static_cast<size_t>(ncimp));
    copyArray(&cimp_keq, t.cimp_keq, ncimp);
    copyArray(&cimp_phase, t.cimp_phase, ncimp);
    copyArray(&cmap_atoms, t.cmap_atoms, 5 * static_cast<size_t>(ncmap));
    copyArray(&cmap_surface, t.cmap_surface, ncmap);
    copyArray(&cmap_dims, t.cmap_dims, ncmap_surf);
    size_t nvalues = 0;
    for (int s = 0; s < ncmap_surf; s++) {
      nvalues += static_cast<size_t>(t.cmap_dims[s]) * t.cmap_dims[s];
    }
    copyArray(&cmap_values, t.cmap_values, nvalues);
    copyArray(&xyz, coords, 3 * n);
    // device memory the molecule holds while in flight: per-atom arrays (coordinates, forces,
    // parameters, GB workspace, minimizer state) on the padded atom count, valence records,
    // Lennard-Jones tables, and per tile its exclusion mask and stored pair derivatives
    const double padded = static_cast<double>((natom + 31) / 32 * 32);
    const double nblk = padded / 32.0;
    bytes = 256.0 * padded + 16.0 * (nbond + nangl + 2.0 * ndihe) + 16.0 * nt2 +
            (128.0 + 8.0 * kPairDerivPerTile) * nblk * (nblk + 1.0) / 2.0 + 1024.0;
  }

  sb_topology view() const {
    sb_topology t;
    std::memset(&t, 0, sizeof(sb_topology));
    t.natom = natom;
    t.charge = ptrOrNull(charge);
    t.lj_idx = ptrOrNull(lj_idx);
    t.n_lj_types = n_lj;
    t.lja = ptrOrNull(lja);
    t.ljb = ptrOrNull(ljb);
    t.lja14 = ptrOrNull(lja14);
    t.ljb14 = ptrOrNull(ljb14);
    t.excl_bounds = ptrOrNull(excl_bounds);
    t.excl_list = ptrOrNull(excl_list);
    t.pb_radii = ptrOrNull(pb_radii);
    t.gb_screen = ptrOrNull(gb_screen);
    t.gb_alpha = ptrOrNull(gb_alpha);
    t.gb_beta = ptrOrNull(gb_beta);
    t.gb_gamma = ptrOrNull(gb_gamma);
    t.nbond = nbond;
    t.bond_atoms = ptrOrNull(bond_atoms);
    t.bond_keq = ptrOrNull(bond_keq);
    t.bond_leq = ptrOrNull(bond_leq);
    t.nangl = nangl;
    t.angl_atoms = ptrOrNull(angl_atoms);
    t.angl_keq = ptrOrNull(angl_keq);
    t.angl_theta0 = ptrOrNull(angl_theta0);
    t.ndihe = ndihe;
    t.dihe_atoms = ptrOrNull(dihe_atoms);
    t.dihe_amp = ptrOrNull(dihe_amp);
    t.dihe_freq = ptrOrNull(dihe_freq);
    t.dihe_phase = ptrOrNull(dihe_phase);
    t.dihe_scee = ptrOrNull(dihe_scee);
    t.dihe_scnb = ptrOrNull(dihe_scnb);
    t.dihe_improper = ptrOrNull(dihe_improper);
    t.nubrd = nubrd;
    t.ubrd_atoms = ptrOrNull(ubrd_atoms);
    t.ubrd_keq = ptrOrNull(ubrd_keq);
    t.ubrd_leq = ptrOrNull(ubrd_leq);
    t.ncimp = ncimp;
    t.cimp_atoms = ptrOrNull(cimp_atoms);
    t.cimp_keq = ptrOrNull(cimp_keq);
    t.cimp_phase = ptrOrNull(cimp_phase);
    t.ncmap = ncmap;
    t.cmap_atoms = ptrOrNull(cmap_atoms);
    t.cmap_surface = ptrOrNull(cmap_surface);
    t.ncmap_surf = ncmap_surf;
    t.cmap_dims = ptrOrNull(cmap_dims);
    t.cmap_values = ptrOrNull(cmap_values);
    return t;
  }
};

struct Result {
  sb_served_result r;
  std::vector<double> xyz;
};

// Admitted requests of one kind running together on one stream: minimizations, or energy and
// force evaluations (one launch)
struct Batch {
  int kind = SB_REQUEST_MINIMIZE;
  std::vector<Request> reqs;
  std::vector<char> finished;
  int remaining = 0;
  double bytes = 0.0;
  cudaStream_t stream = nullptr;
  cudaEvent_t event = nullptr;
  std::unique_ptr<Synthesis> syn;
};

}  // namespace

class Server {
public:
  explicit Server(const sb_server_options &o) : opt_(o), t0_(std::chrono::steady_clock::now()) {
    if (!(o.hbm_budget_bytes > 0.0) || o.max_batch_molecules < 1 || o.max_batches < 1 ||
        o.cycles_per_launch < 1) {
      throw Error(SB_ERR_ARGUMENT, "server budget, batch limits and cycles per launch must be "
                  "positive");
    }
    if (!(o.migrate_fraction >= 0.0 && o.migrate_fraction < 1.0)) {
      throw Error(SB_ERR_ARGUMENT, "migrate_fraction must lie in [0, 1)");
    }
    validateMinimizeControls(o.controls);
    if (o.options.precision != SB_PRECISION_SINGLE && o.options.precision != SB_PRECISION_DOUBLE) {
      throw Error(SB_ERR_ARGUMENT, "precision must be SB_PRECISION_SINGLE or SB_PRECISION_DOUBLE");
    }
    if (o.options.precision == SB_PRECISION_DOUBLE && o.controls.kernel != SB_MIN_GRAPH) {
      throw Error(SB_ERR_UNSUPPORTED, "an FP64 server minimizes with the graph minimizer: set "
                  "controls.kernel to SB_MIN_GRAPH");
    }
    int ndev = 0;
    cudaCheck(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (o.options.device < 0 || o.options.device >= ndev) {
      throw Error(SB_ERR_DEVICE, "CUDA device " + std::to_string(o.options.device) +
                  " not present");
    }
    worker_ = std::thread([this]() { this->run(); });
  }

  ~Server() {
    {
      std::lock_guard<std::mutex> lock(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) {
      worker_.join();
    }
  }

  long long submit(const sb_topology* top, const double* xyz, int kind) {
    if (top == nullptr || xyz == nullptr || top->natom <= 0) {
      throw Error(SB_ERR_ARGUMENT, "a request needs a topology with atoms and coordinates");
    }
    if (kind != SB_REQUEST_MINIMIZE && kind != SB_REQUEST_EVALUATE) {
      throw Error(SB_ERR_ARGUMENT, "unknown request kind " + std::to_string(kind));
    }
    validateTopology(*top, opt_.options, -1);
    const int on_chip = (opt_.options.tiled_above_atoms > 0) ? opt_.options.tiled_above_atoms : 2048;
    if (kind == SB_REQUEST_MINIMIZE && top->natom > on_chip &&
        opt_.controls.kernel != SB_MIN_GRAPH) {
      throw Error(SB_ERR_UNSUPPORTED, "molecules above " + std::to_string(on_chip) +
                  " atoms are evaluated tile by tile and cannot be minimized by the persistent "
                  "kernel; a server whose controls select SB_MIN_GRAPH minimizes them");
    }
    if (kind == SB_REQUEST_MINIMIZE && (top->nubrd > 0 || top->ncimp > 0 || top->ncmap > 0) &&
        opt_.controls.kernel != SB_MIN_GRAPH) {
      throw Error(SB_ERR_UNSUPPORTED, "CHARMM terms cannot be minimized by the persistent "
                  "kernel; a server whose controls select SB_MIN_GRAPH minimizes them");
    }
    Request req(*top, xyz);
    req.kind = kind;
    if (opt_.options.precision == SB_PRECISION_DOUBLE) {
      req.bytes *= 2.0;   // the FP64 mode's per-atom and per-term arrays are twice as wide
    }
    if (req.bytes > opt_.hbm_budget_bytes) {
      throw Error(SB_ERR_ARGUMENT, "the molecule alone exceeds the server's HBM budget");
    }
    std::lock_guard<std::mutex> lock(mu_);
    failIfBroken();
    req.id = next_id_++;
    req.t_submit = now();
    const long long id = req.id;
    pending_.push_back(std::move(req));
    submitted_++;
    cv_.notify_all();
    return id;
  }

  int poll(sb_served_result* out, int max_results, double* xyz, long long cap) {
    std::lock_guard<std::mutex> lock(mu_);
    if (results_.empty()) {
      failIfBroken();
    }
    int n = 0;
    long long used = 0;
    while (n < max_results && !results_.empty()) {
      const Result &r = results_.front();
      const long long need = static_cast<long long>(r.xyz.size());
      if (xyz != nullptr) {
        if (used + need > cap) {
          break;
        }
        if (need > 0) {
          std::memcpy(xyz + used, r.xyz.data(), sizeof(double) * need);
        }
        used += need;
      }
      out[n++] = r.r;
      results_.pop_front();
    }
    return n;
  }

  bool drain(double timeout) {
    std::unique_lock<std::mutex> lock(mu_);
    const auto until = std::chrono::steady_clock::now() +
                       std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                           std::chrono::duration<double>(timeout));
    while (!idle() && error_.empty()) {
      if (idle_cv_.wait_until(lock, until) == std::cv_status::timeout) {
        break;
      }
    }
    failIfBroken();
    return idle();
  }

  sb_server_stats stats() {
    std::lock_guard<std::mutex> lock(mu_);
    sb_server_stats s;
    s.submitted = submitted_;
    s.admitted = admitted_;
    s.completed = completed_;
    s.failed = failed_;
    s.migrated = migrated_;
    s.pending = static_cast<int>(pending_.size());
    s.in_flight = in_flight_;
    s.batches = nbatches_;
    s.bytes_in_flight = bytes_in_flight_;
    return s;
  }

private:
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count();
  }

  // Nothing queued, in flight or holding device memory (called with mu_ held)
  bool idle() const {
    return pending_.empty() && in_flight_ == 0 && nbatches_ == 0;
  }

  void failIfBroken() const {
    if (!error_.empty()) {
      throw Error(SB_ERR_CUDA, "server worker stopped: " + error_);
    }
  }

  // After an error: clear it if it does not persist, and throw if the CUDA context is lost (an
  // event that was never recorded queries as complete unless the context has failed)
  void checkContext() {
    cudaGetLastError();
    const cudaError_t e = cudaEventQuery(probe_);
    if (e != cudaSuccess) {
      throw Error(SB_ERR_CUDA, std::string("CUDA context lost: ") + cudaGetErrorString(e));
    }
  }

  // Requests admitted in arrival order while the batch and the memory budget allow: the oldest
  // pending request's kind only; a request retried alone after a failed build forms a batch of
  // its own.  Called with mu_ held.
  std::vector<Request> takePending() {
    std::vector<Request> take;
    const int kind = pending_.front().kind;
    double bytes = bytes_in_flight_;
    for (auto it = pending_.begin(); it != pending_.end() &&
         static_cast<int>(take.size()) < opt_.max_batch_molecules;) {
      if (it->kind != kind) {
        ++it;
        continue;
      }
      if (bytes + it->bytes > opt_.hbm_budget_bytes || (it->solo && !take.empty())) {
        break;
      }
      const bool solo = it->solo;
      bytes += it->bytes;
      take.push_back(std::move(*it));
      it = pending_.erase(it);
      if (solo) {
        break;
      }
    }
    if (!take.empty()) {
      bytes_in_flight_ = bytes;
      in_flight_ += static_cast<int>(take.size());
      admitted_ += static_cast<long long>(take.size());
      nbatches_++;
    }
    return take;
  }

  void run() {
    std::vector<std::unique_ptr<Batch>> batches;
    try {
      cudaCheck(cudaSetDevice(opt_.options.device), "cudaSetDevice");
      cudaCheck(cudaEventCreateWithFlags(&probe_, cudaEventDisableTiming), "cudaEventCreate");
      while (true) {
        bool progress = false;
        for (size_t b = 0; b < batches.size();) {
          const cudaError_t q = cudaEventQuery(batches[b]->event);
          if (q == cudaErrorNotReady) {
            b++;
            continue;
          }
          progress = true;
          bool finished = false;
          try {
            cudaCheck(q, "batch launch");
            finished = service(batches[b].get());
          }
          catch (const Error &e) {
            // this batch's requests fail; the other batches carry on unless the context is lost
            std::unique_ptr<Batch> failed = std::move(batches[b]);
            batches.erase(batches.begin() + b);
            failBatch(std::move(failed), e.code);
            checkContext();
            continue;
          }
          if (finished) {
            retire(std::move(batches[b]));
            batches.erase(batches.begin() + b);
          }
          else {
            b++;
          }
        }
        std::vector<Request> take;
        {
          std::unique_lock<std::mutex> lock(mu_);
          if (stop_) {
            break;
          }
          if (static_cast<int>(batches.size()) < opt_.max_batches && !pending_.empty()) {
            take = takePending();
          }
          if (take.empty() && !progress) {
            // nothing to launch or collect: sleep until a submission or a short timeout
            cv_.wait_for(lock, std::chrono::microseconds(batches.empty() ? 2000 : 100));
            continue;
          }
        }
        if (!take.empty()) {
          std::unique_ptr<Batch> b = makeBatch(std::move(take));
          try {
            start(b.get());
            batches.push_back(std::move(b));
          }
          catch (const Error &e) {
            if (b->reqs.size() > 1) {
              requeueAlone(std::move(b));
            }
            else {
              failBatch(std::move(b), e.code);
            }
            checkContext();
          }
        }
      }
      // stop: let the launches in flight finish, then release every batch on its stream
      for (auto &b : batches) {
        cudaEventSynchronize(b->event);
        retire(std::move(b));
      }
    }
    catch (const std::exception &e) {
      // the context is lost (or the worker could not start): return what is in flight as failed
      for (auto &b : batches) {
        if (b) {
          failBatch(std::move(b), SB_ERR_CUDA);
        }
      }
      std::lock_guard<std::mutex> lock(mu_);
      error_ = e.what();
      idle_cv_.notify_all();
    }
    if (probe_ != nullptr) {
      cudaEventDestroy(probe_);
      probe_ = nullptr;
    }
  }

  std::unique_ptr<Batch> makeBatch(std::vector<Request> take) {
    auto b = std::make_unique<Batch>();
    b->kind = take.front().kind;
    b->reqs = std::move(take);
    b->finished.assign(b->reqs.size(), 0);
    b->remaining = static_cast<int>(b->reqs.size());
    for (const Request &r : b->reqs) {
      b->bytes += r.bytes;
    }
    return b;
  }

  // Build, upload and start a batch on a stream of its own
  void start(Batch* b) {
    cudaCheck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    cudaCheck(cudaEventCreateWithFlags(&b->event, cudaEventDisableTiming), "cudaEventCreate");
    const double t = now();
    std::vector<sb_topology> tops;
    std::vector<int> index;
    std::vector<double> xyz;
    for (size_t k = 0; k < b->reqs.size(); k++) {
      Request &r = b->reqs[k];
      if (r.state == nullptr) {
        r.t_admit = t;
      }
      tops.push_back(r.view());
      index.push_back(static_cast<int>(k));
      xyz.insert(xyz.end(), r.xyz.begin(), r.xyz.end());
    }
    {
      AllocationStreamGuard guard(b->stream);
      b->syn = std::make_unique<Synthesis>(tops.data(), static_cast<int>(tops.size()),
                                           index.data(), static_cast<int>(tops.size()),
                                           opt_.options);
      b->syn->setCoordinates(xyz.data(), b->stream);
      if (b->kind == SB_REQUEST_MINIMIZE) {
        b->syn->minimizeBegin(opt_.controls, b->stream);
        // molecules moved here from an emptying batch continue from their own state
        for (size_t k = 0; k < b->reqs.size(); k++) {
          if (b->reqs[k].state != nullptr) {
            b->syn->importMinimizerState(static_cast<int>(k), *b->reqs[k].state, b->stream);
            b->reqs[k].state.reset();
          }
        }
      }
    }
    if (b->kind == SB_REQUEST_MINIMIZE) {
      b->syn->minimizeAdvance(opt_.cycles_per_launch, true, b->stream);
    }
    else {
      b->syn->initialize(SB_INIT_FORCES | SB_INIT_ENERGIES | SB_INIT_GB_WORKSPACE, b->stream);
      b->syn->evaluate(SB_TERM_ALL, true, true, b->stream);
    }
    cudaCheck(cudaEventRecord(b->event, b->stream), "cudaEventRecord");
  }

  // A batch that could not be built: release it and queue its requests again, at the front in
  // their order, each to be admitted alone
  void requeueAlone(std::unique_ptr<Batch> b) {
    std::vector<Request> reqs = std::move(b->reqs);
    b->reqs.clear();
    retire(std::move(b));
    std::lock_guard<std::mutex> lock(mu_);
    in_flight_ -= static_cast<int>(reqs.size());
    admitted_ -= static_cast<long long>(reqs.size());
    for (auto it = reqs.rbegin(); it != reqs.rend(); ++it) {
      it->solo = true;
      pending_.push_front(std::move(*it));
    }
    cv_.notify_all();
  }

  // The unfinished requests of a batch are returned with the error code; the batch is released
  void failBatch(std::unique_ptr<Batch> b, int code) {
    const double t = now();
    std::vector<Result> out;
    for (size_t k = 0; k < b->reqs.size(); k++) {
      if (b->finished[k]) {
        continue;
      }
      const Request &r = b->reqs[k];
      Result res;
      std::memset(&res.r, 0, sizeof(sb_served_result));
      res.r.request_id = r.id;
      res.r.natom = r.natom;
      res.r.kind = r.kind;
      res.r.status = (code != SB_OK) ? code : SB_ERR_CUDA;
      res.r.energy = std::nan("");
      res.r.rms_force = std::nan("");
      res.r.submit_time = r.t_submit;
      res.r.admit_time = r.t_admit;
      res.r.finish_time = t;
      out.push_back(std::move(res));
      b->finished[k] = 1;
    }
    b->remaining = 0;
    retire(std::move(b));
    std::lock_guard<std::mutex> lock(mu_);
    for (auto &res : out) {
      results_.push_back(std::move(res));
    }
    in_flight_ -= static_cast<int>(out.size());
    completed_ += static_cast<long long>(out.size());
    failed_ += static_cast<long long>(out.size());
    if (idle()) {
      idle_cv_.notify_all();
    }
  }

  // Results of an evaluation batch (all of it completes with its one launch)
  void serviceEvaluation(Batch* b) {
    const int n = static_cast<int>(b->reqs.size());
    std::vector<double> nrg(static_cast<size_t>(n) * SB_NRG_STRIDE);
    std::vector<double> frc(3 * static_cast<size_t>(b->syn->natom_total));
    b->syn->getEnergies(nrg.data(), b->stream);
    b->syn->getForces(frc.data(), b->stream);
    const double t = now();
    std::vector<Result> out;
    size_t off = 0;
    for (int k = 0; k < n; k++) {
      const Request &r = b->reqs[k];
      Result res;
      std::memset(&res.r, 0, sizeof(sb_served_result));
      res.r.request_id = r.id;
      res.r.natom = r.natom;
      res.r.kind = SB_REQUEST_EVALUATE;
      double total = 0.0, f2 = 0.0;
      for (int q = 0; q < SB_NRG_STRIDE; q++) {
        res.r.energies[q] = nrg[static_cast<size_t>(k) * SB_NRG_STRIDE + q];
        total += res.r.energies[q];
      }
      const size_t len = 3 * static_cast<size_t>(r.natom);
      for (size_t q = 0; q < len; q++) {
        f2 += frc[off + q] * frc[off + q];
      }
      res.r.energy = total;
      res.r.rms_force = std::sqrt(f2 / static_cast<double>(len));
      res.r.submit_time = r.t_submit;
      res.r.admit_time = r.t_admit;
      res.r.finish_time = t;
      res.xyz.assign(frc.begin() + off, frc.begin() + off + len);
      off += len;
      out.push_back(std::move(res));
      b->finished[k] = 1;
    }
    b->remaining = 0;
    std::lock_guard<std::mutex> lock(mu_);
    for (auto &res : out) {
      results_.push_back(std::move(res));
    }
    in_flight_ -= n;
    completed_ += n;
    if (idle()) {
      idle_cv_.notify_all();
    }
  }

  // After a launch of the batch finished: retire what is done, relaunch the rest.  Returns true
  // when every molecule of the batch has retired.
  bool service(Batch* b) {
    if (b->kind == SB_REQUEST_EVALUATE) {
      serviceEvaluation(b);
      return true;
    }
    const int n = static_cast<int>(b->reqs.size());
    std::vector<int> cycles(n), done(n);
    std::vector<double> rms(n);
    b->syn->getMinimizeProgress(cycles.data(), done.data(), rms.data(), b->stream);
    std::vector<int> newly;
    for (int k = 0; k < n; k++) {
      if (!b->finished[k] && (done[k] || cycles[k] >= opt_.controls.total_cycles)) {
        newly.push_back(k);
      }
    }
    if (!newly.empty()) {
      std::vector<double> nrg(static_cast<size_t>(n) * SB_NRG_STRIDE);
      std::vector<double> xyz(3 * static_cast<size_t>(b->syn->natom_total));
      b->syn->getEnergies(nrg.data(), b->stream);
      b->syn->getCoordinates(xyz.data(), b->stream);
      const double t = now();
      std::vector<size_t> first(n + 1, 0);   // unpadded atom offsets, systems in batch order
      for (int k = 0; k < n; k++) {
        first[k + 1] = first[k] + static_cast<size_t>(b->reqs[k].natom);
      }
      std::vector<Result> out;
      for (int k : newly) {
        const Request &r = b->reqs[k];
        Result res;
        std::memset(&res.r, 0, sizeof(sb_served_result));
        res.r.request_id = r.id;
        res.r.natom = r.natom;
        res.r.cycles = cycles[k];
        res.r.converged = done[k];
        res.r.rms_force = rms[k];
        res.r.kind = SB_REQUEST_MINIMIZE;
        double total = 0.0;
        for (int q = 0; q < SB_NRG_STRIDE; q++) {
          res.r.energies[q] = nrg[static_cast<size_t>(k) * SB_NRG_STRIDE + q];
          total += res.r.energies[q];
        }
        res.r.energy = total;
        res.r.submit_time = r.t_submit;
        res.r.admit_time = r.t_admit;
        res.r.finish_time = t;
        const size_t off = 3 * first[k];
        res.xyz.assign(xyz.begin() + off, xyz.begin() + off + 3 * static_cast<size_t>(r.natom));
        out.push_back(std::move(res));
        b->finished[k] = 1;
        b->remaining--;
      }
      std::lock_guard<std::mutex> lock(mu_);
      for (auto &res : out) {
        results_.push_back(std::move(res));
      }
      in_flight_ -= static_cast<int>(newly.size());
      completed_ += static_cast<long long>(newly.size());
      if (pending_.empty() && in_flight_ == 0) {
        idle_cv_.notify_all();
      }
    }
    if (b->remaining == 0) {
      return true;
    }
    if (shouldMigrate(b)) {
      migrate(b);
      return true;
    }
    b->syn->minimizeAdvance(opt_.cycles_per_launch, true, b->stream);
    cudaCheck(cudaEventRecord(b->event, b->stream), "cudaEventRecord");
    return false;
  }

  // A minimization batch whose molecules have mostly retired holds its whole memory budget and
  // a launch per round for the few left.  When minimizations are waiting, those few move to
  // the front of the queue with their minimizer state, the batch is released, and they are
  // admitted again beside the waiting requests: their slots are backfilled.  Each moved
  // molecule continues exactly where it was (state at a cycle boundary, the persistent FP32
  // minimizer, whose per-molecule arithmetic does not depend on the batch).
  bool shouldMigrate(const Batch* b) {
    if (opt_.controls.kernel != SB_MIN_PERSISTENT ||
        opt_.options.precision != SB_PRECISION_SINGLE || b->reqs.size() < 2 ||
        static_cast<double>(b->remaining) >
            opt_.migrate_fraction * static_cast<double>(b->reqs.size())) {
      return false;
    }
    std::lock_guard<std::mutex> lock(mu_);
    for (const Request &r : pending_) {
      if (r.kind == SB_REQUEST_MINIMIZE && r.state == nullptr) {
        return true;
      }
    }
    return false;
  }

  void migrate(Batch* b) {
    std::vector<Request> moving;
    for (size_t k = 0; k < b->reqs.size(); k++) {
      if (b->finished[k]) {
        continue;
      }
      auto st = std::make_shared<MinimizerState>();
      b->syn->exportMinimizerState(static_cast<int>(k), st.get(), b->stream);
      Request r = std::move(b->reqs[k]);
      r.state = std::move(st);
      moving.push_back(std::move(r));
      b->finished[k] = 1;
    }
    b->remaining = 0;
    std::lock_guard<std::mutex> lock(mu_);
    in_flight_ -= static_cast<int>(moving.size());
    admitted_ -= static_cast<long long>(moving.size());
    migrated_ += static_cast<long long>(moving.size());
    for (auto it = moving.rbegin(); it != moving.rend(); ++it) {
      pending_.push_front(std::move(*it));
    }
    cv_.notify_all();
  }

  // Free a batch's device memory in its stream's order, then its stream
  void retire(std::unique_ptr<Batch> b) {
    if (b->stream != nullptr) {
      AllocationStreamGuard guard(b->stream);
      b->syn.reset();
    }
    else {
      b->syn.reset();
    }
    if (b->event != nullptr) {
      cudaEventDestroy(b->event);
    }
    if (b->stream != nullptr) {
      cudaStreamDestroy(b->stream);
    }
    std::lock_guard<std::mutex> lock(mu_);
    bytes_in_flight_ -= b->bytes;
    if (bytes_in_flight_ < 0.0) {
      bytes_in_flight_ = 0.0;
    }
    nbatches_--;
    cv_.notify_all();
    if (idle()) {
      idle_cv_.notify_all();
    }
  }

  sb_server_options opt_;
  std::chrono::steady_clock::time_point t0_;
  std::thread worker_;
  std::mutex mu_;
  std::condition_variable cv_;        // worker wake-up: submissions, stop
  std::condition_variable idle_cv_;   // drain: nothing queued or in flight
  std::deque<Request> pending_;
  std::deque<Result> results_;
  long long next_id_ = 1;
  long long submitted_ = 0;
  long long admitted_ = 0;
  long long completed_ = 0;
  long long failed_ = 0;
  long long migrated_ = 0;
  int in_flight_ = 0;
  int nbatches_ = 0;
  double bytes_in_flight_ = 0.0;
  bool stop_ = false;
  std::string error_;
  cudaEvent_t probe_ = nullptr;       // never recorded: queries fail only with a lost context
};

}  // namespace sb

// ------------------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------------------
struct sb_server {
  std::unique_ptr<sb::Server> impl;
};

namespace {

template <typename F> int serverGuarded(F &&f) {
  try {
    f();
    return SB_OK;
  }
  catch (const sb::Error &e) {
    sb::setLastError(e.what());
    return e.code;
  }
  catch (const std::exception &e) {
    sb::setLastError(e.what());
    return SB_ERR_ARGUMENT;
  }
}

sb::Server* needServer(sb_server* s) {
  if (s == nullptr || !s->impl) {
    throw sb::Error(SB_ERR_ARGUMENT, "null server handle");
  }
  return s->impl.get();
}

}  // namespace

extern "C" {

void sb_default_server_options(sb_server_options* opt) {
  std::memset(opt, 0, sizeof(sb_server_options));
  sb_default_options(&opt->options);
  sb_default_minimize_controls(&opt->controls);
  opt->controls.total_cycles = 2000;
  opt->controls.convergence_rms = 0.01;
  // small batches: the persistent kernel's on-chip cycles beat per-cycle graph launches
  opt->controls.kernel = SB_MIN_PERSISTENT;
  opt->hbm_budget_bytes = 2.0e9;
  opt->max_batch_molecules = 512;
  opt->max_batches = 16;
  opt->cycles_per_launch = 50;
  opt->migrate_fraction = 0.25;
}

int sb_server_create(const sb_server_options* opt, sb_server** out) {
  return serverGuarded([&]() {
    if (out == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null output handle");
    *out = nullptr;
    sb_server_options o;
    if (opt != nullptr) {
      o = *opt;
    }
    else {
      sb_default_server_options(&o);
    }
    auto h = std::make_unique<sb_server>();
    h->impl = std::make_unique<sb::Server>(o);
    *out = h.release();
  });
}

int sb_server_submit(sb_server* srv, const sb_topology* top, const double* xyz,
                     long long* request_id) {
  return serverGuarded([&]() {
    const long long id = needServer(srv)->submit(top, xyz, SB_REQUEST_MINIMIZE);
    if (request_id) *request_id = id;
  });
}

int sb_server_submit_evaluation(sb_server* srv, const sb_topology* top, const double* xyz,
                                long long* request_id) {
  return serverGuarded([&]() {
    const long long id = needServer(srv)->submit(top, xyz, SB_REQUEST_EVALUATE);
    if (request_id) *request_id = id;
  });
}

int sb_server_poll(sb_server* srv, sb_served_result* results, int max_results, double* xyz,
                   long long xyz_capacity, int* count) {
  return serverGuarded([&]() {
    if (results == nullptr && max_results > 0) {
      throw sb::Error(SB_ERR_ARGUMENT, "null result array");
    }
    const int n = needServer(srv)->poll(results, max_results, xyz, xyz_capacity);
    if (count) *count = n;
  });
}

int sb_server_drain(sb_server* srv, double timeout_seconds) {
  bool drained = false;
  const int rc = serverGuarded([&]() { drained = needServer(srv)->drain(timeout_seconds); });
  if (rc != SB_OK) return rc;
  return drained ? SB_OK : SB_TIMEOUT;
}

int sb_server_get_stats(sb_server* srv, sb_server_stats* stats) {
  return serverGuarded([&]() {
    if (stats == nullptr) throw sb::Error(SB_ERR_ARGUMENT, "null stats");
    *stats = needServer(srv)->stats();
  });
}

int sb_server_destroy(sb_server* srv) {
  return serverGuarded([&]() { delete srv; });
}

}  // extern "C"
