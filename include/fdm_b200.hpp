/* C++ host class over the C ABI of include/fdm_b200.h: the reference's operator API for the fast fiber path.
 *
 * fdm::FastMonodomainSolver has the method names and meaning of the reference's FastMonodomainSolverBase
 * (core/src/specialized_solver/fast_monodomain_solver/fast_monodomain_solver_base.h:85-124): initialize, run,
 * advanceTimeSpan, setTimeSpan, startTime, endTime, data, reset, callOutputWriter,
 * saveFiberDataCheckpoint, restoreFiberDataCheckpoint.  advanceTimeSpan over [startTime, endTime] is the
 * RepeatedCall loop that drives it in the reference (core/src/control/repeated_call.tpp:43-80).  It is built
 * from fdm::FiberSettings -- the parsed settings (the fiber geometry, the CellML parameters and initial
 * states, the stimulation tables and the time step widths) -- not from PETSc objects; FiberSettings::load
 * reads the file opendihu_b200.solver.write_host_settings writes from a reference settings dict.
 * Errors are fdm::Error exceptions carrying the library's status code and message.
 * Header only; link with -lfdm_b200 (opendihu_b200/libfdm_b200.so). */
#ifndef FDM_B200_HPP
#define FDM_B200_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fdm_b200.h"

namespace fdm {

class Error : public std::runtime_error {
 public:
  Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
  int code() const { return code_; }

 private:
  int code_;
};

/* Page-locked host memory (fdm_host_alloc) for std::vector: state arrays in it are transferred by DMA without
 * staging, e.g. std::vector<double, fdm::PinnedAllocator<double>> states(nStates * nNodes). */
template<class T>
struct PinnedAllocator {
  using value_type = T;
  PinnedAllocator() = default;
  template<class U>
  PinnedAllocator(const PinnedAllocator<U>&) {}
  T* allocate(size_t n)
  {
    void* p = nullptr;
    const int rc = fdm_host_alloc(n * sizeof(T), &p);
    if (rc != FDM_OK) {
      const char* m = fdm_last_error(nullptr);
      throw Error(rc, m ? m : "fdm_host_alloc failed");
    }
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t) { fdm_host_free(p); }
  template<class U>
  bool operator==(const PinnedAllocator<U>&) const { return true; }
  template<class U>
  bool operator!=(const PinnedAllocator<U>&) const { return false; }
};

/* The parsed settings of one FastMonodomainSolver (all fibers of the rank). */
struct FiberSettings {
  fdm_config config{};                       // model, schemes, method, precision, time step widths, options
  double start_time = 0.0, end_time = 0.0;   // RepeatedCall startTime / endTime
  std::vector<int64_t> fiber_offsets;        // n_fibers + 1 node offsets
  std::vector<double> element_lengths;       // per fiber n_f - 1 lengths, concatenated
  std::vector<double> prefactor;             // per fiber sigma / (Am Cm)
  std::vector<double> parameters;            // [parameter][node] (empty: the model's defaults)
  std::vector<double> states;                // [state][node] (empty: the model's initial values)
  std::vector<uint8_t> firing_events;        // [row][motor unit]
  int firing_rows = 0, firing_cols = 0;
  std::vector<int> motor_unit_no, stimulation_point_index;
  std::vector<double> call_frequency, repeat_after_first_call, call_enable_begin;
  std::vector<double> jitter;                // [fiber][k]
  int n_jitter = 0;
  std::vector<int> algebraics_for_transfer, states_for_transfer{0};
  std::vector<int> fiber_numbers;            // global fiber numbers ("additionalArgument"; empty: the index)
  bool initialize_states_to_equilibrium = false;  // "initializeStatesToEquilibrium" of the CellML settings
  double equilibrium_dt = 1e-4;                   // "initializeStatesToEquilibriumTimestepWidth"

  int n_fibers() const { return fiber_offsets.empty() ? 0 : (int)fiber_offsets.size() - 1; }
  int64_t n_nodes() const { return fiber_offsets.empty() ? 0 : fiber_offsets.back(); }

  /* Reads "key count value..." lines (the format write_host_settings writes; '#' starts a comment). */
  static FiberSettings load(const std::string& path)
  {
    std::ifstream in(path);
    if (!in)
      throw Error(FDM_ERR_ARG, "fdm::FiberSettings::load: cannot open " + path);
    std::map<std::string, std::vector<double>> kv;
    std::string line;
    while (std::getline(in, line)) {
      if (line.empty() || line[0] == '#')
        continue;
      std::istringstream ls(line);
      std::string key;
      long long count = 0;
      if (!(ls >> key >> count) || count < 0)
        throw Error(FDM_ERR_ARG, "fdm::FiberSettings::load: bad line: " + line.substr(0, 80));
      std::vector<double> v((size_t)count);
      for (auto& x : v)
        if (!(ls >> x))
          throw Error(FDM_ERR_ARG, "fdm::FiberSettings::load: too few values for " + key);
      kv[key] = std::move(v);
    }
    FiberSettings s;
    fdm_config_default(&s.config);
    auto has = [&](const char* k) { return kv.count(k) > 0; };
    auto num = [&](const char* k) -> double {
      auto it = kv.find(k);
      if (it == kv.end() || it->second.size() != 1)
        throw Error(FDM_ERR_ARG, std::string("fdm::FiberSettings::load: missing scalar ") + k);
      return it->second[0];
    };
    auto vec = [&](const char* k) -> const std::vector<double>& {
      static const std::vector<double> empty;
      auto it = kv.find(k);
      return it == kv.end() ? empty : it->second;
    };
    auto as_int = [&](const char* k) {
      std::vector<int> o;
      for (double x : vec(k))
        o.push_back((int)x);
      return o;
    };
    fdm_config& c = s.config;
    c.model = (int)num("model");
    c.diffusion_scheme = (int)num("diffusion_scheme");
    c.method = (int)num("method");
    c.reaction_precision = (int)num("reaction_precision");
    c.approximate_exponential_function = (int)num("approximate_exponential_function");
    c.clamp_rule = (int)num("clamp_rule");
    c.vc_width = (int)num("vc_width");
    c.n_ranks = (int)num("n_ranks");
    c.stimulus_mode = (int)num("stimulus_mode");
    c.stimulus_parameter = (int)num("stimulus_parameter");
    c.stimulus_value = num("stimulus_value");
    c.value_for_stimulated_point = num("value_for_stimulated_point");
    c.dt_repeated_call = num("dt_repeated_call");
    c.dt_splitting = num("dt_splitting");
    c.dt_0d = num("dt_0d");
    c.dt_1d = num("dt_1d");
    c.only_compute_if_stimulated = (int)num("only_compute_if_stimulated");
    c.skip_close_to_equilibrium = (int)num("skip_close_to_equilibrium");
    if (has("device"))
      c.device = (int)num("device");
    s.start_time = num("start_time");
    s.end_time = num("end_time");
    for (double x : vec("fiber_offsets"))
      s.fiber_offsets.push_back((int64_t)x);
    s.element_lengths = vec("element_lengths");
    s.prefactor = vec("prefactor");
    s.parameters = vec("parameters");
    s.states = vec("states");
    for (double x : vec("firing_events"))
      s.firing_events.push_back((uint8_t)x);
    s.firing_rows = (int)num("firing_rows");
    s.firing_cols = (int)num("firing_cols");
    s.motor_unit_no = as_int("motor_unit_no");
    s.stimulation_point_index = as_int("stimulation_point_index");
    s.call_frequency = vec("call_frequency");
    s.repeat_after_first_call = vec("repeat_after_first_call");
    s.call_enable_begin = vec("call_enable_begin");
    s.jitter = vec("jitter");
    s.n_jitter = (int)num("n_jitter");
    s.algebraics_for_transfer = as_int("algebraics_for_transfer");
    if (has("states_for_transfer"))
      s.states_for_transfer = as_int("states_for_transfer");
    s.fiber_numbers = as_int("fiber_numbers");
    if (has("initialize_states_to_equilibrium"))
      s.initialize_states_to_equilibrium = num("initialize_states_to_equilibrium") != 0;
    if (has("equilibrium_dt"))
      s.equilibrium_dt = num("equilibrium_dt");
    return s;
  }
};

/* One entry of the stimulation log (StimulationLogging::StimulationLogEntry, stimulation_logging.h:28-33). */
struct StimulationLogEntry {
  double time;
  int motorUnitNo;
  int fiberNo;
};

/* The transferred fiber data (updateFiberData: statesForTransfer, algebraicsForTransfer), [k][node]. */
struct TransferData {
  std::vector<double> vm;
  std::vector<double> states;      // statesForTransfer[1..]
  std::vector<double> algebraics;  // algebraicsForTransfer
};

/* One output writer of the diffusion solver.  When it writes restates OutputWriter::Generic::prepareWrite
 * (core/src/output_writer/generic.tpp:14-115): every call adds callCountIncrement to a call counter, a call
 * writes when the counter passes a multiple of outputInterval (or its increment is 0: the initial values),
 * under <filename>_<no:07d>, no being the running file number or, with timeStepIndexNumbering, the counter.
 * What is written is the callback's: it gets the numbered name and the current time, and reads the fiber
 * data through FastMonodomainSolver::data(). */
struct OutputWriter {
  int outputInterval = 1;
  std::string filename = "out";
  bool timeStepIndexNumbering = false;
  std::function<void(const std::string& name, double currentTime)> write;
  int writeCallCount = 0;
  int outputFileNo = 0;

  /* counts one call; true (and the numbered name) when it writes */
  bool prepare(int timeStepNo, int callCountIncrement, std::string& name)
  {
    const int interval = outputInterval > 0 ? outputInterval : 1;
    const int old = writeCallCount;
    writeCallCount += callCountIncrement;
    const int last = writeCallCount - writeCallCount % interval;
    if (!((old < last && last <= writeCallCount) || callCountIncrement == 0))
      return false;
    name = filename;
    if (timeStepNo != -1) {
      char no[16];
      std::snprintf(no, sizeof(no), "_%07d", timeStepIndexNumbering ? writeCallCount : outputFileNo);
      name += no;
    }
    outputFileNo++;
    return true;
  }
};

class FastMonodomainSolver {
 public:
  explicit FastMonodomainSolver(FiberSettings settings) : s_(std::move(settings))
  {
    start_ = s_.start_time;
    end_ = s_.end_time;
    current_time_ = s_.start_time;
  }
  FastMonodomainSolver(const FastMonodomainSolver&) = delete;
  FastMonodomainSolver& operator=(const FastMonodomainSolver&) = delete;
  FastMonodomainSolver(FastMonodomainSolver&& o) noexcept
      : s_(std::move(o.s_)), h_(o.h_), start_(o.start_), end_(o.end_), writers_(std::move(o.writers_)),
        current_time_(o.current_time_), piece_steps_(o.piece_steps_), log_on_(o.log_on_),
        equilibrium_done_(o.equilibrium_done_), equilibrium_iterations_(o.equilibrium_iterations_)
  {
    o.h_ = nullptr;
  }
  ~FastMonodomainSolver() { reset(); }

  void initialize()
  {
    if (h_)
      return;
    fdm_solver* h = nullptr;
    int rc = fdm_create(&s_.config, &h);
    if (rc != FDM_OK)
      throw Error(rc, std::string("fdm_create: ") + fdm_last_error(nullptr));
    h_ = h;
    try {
      const int nf = s_.n_fibers();
      if (s_.initialize_states_to_equilibrium && !equilibrium_done_)
        initialize_to_equilibrium();
      check(fdm_set_fibers(h_, nf, s_.fiber_offsets.data(), s_.element_lengths.data(), s_.prefactor.data()));
      if (!s_.parameters.empty())
        check(fdm_set_parameters(h_, s_.parameters.data()));
      if (!s_.states.empty())
        check(fdm_set_states(h_, s_.states.data()));
      const double zero = 0.0;
      check(fdm_set_stimulation(h_, s_.firing_events.data(), s_.firing_rows, s_.firing_cols,
                                s_.motor_unit_no.data(), s_.stimulation_point_index.data(), s_.call_frequency.data(),
                                s_.repeat_after_first_call.data(), s_.call_enable_begin.data(),
                                s_.jitter.empty() ? &zero : s_.jitter.data(), s_.n_jitter));
      if (!s_.algebraics_for_transfer.empty())
        check(fdm_set_algebraics_for_transfer(h_, (int)s_.algebraics_for_transfer.size(),
                                              s_.algebraics_for_transfer.data()));
    } catch (...) {
      reset();
      throw;
    }
  }

  void run()
  {
    initialize();
    advanceTimeSpan();
  }

  /* RepeatedCall over [startTime, endTime].  The output writers run after every RepeatedCall piece, as the
   * reference's advanceTimeSpan calls the diffusion's writers (fast_monodomain_solver_compute.tpp:35-44) with
   * timeStepNo 0, the piece's end time and its number of split steps: the advance stops only after the
   * pieces whose call writes, the steps stay those of one advance over the span (fdm_advance_pieces). */
  void advanceTimeSpan(bool withOutputWritersEnabled = true)
  {
    initialize();
    if (log_on_)
      grow_stimulation_log(end_ - start_);
    int64_t n = 0;
    check(fdm_repeated_call_plan(h_, start_, end_, &n, nullptr));
    std::vector<int> steps((size_t)(n > 0 ? n : 1), 0);
    if (!writers_.empty())
      check(fdm_repeated_call_plan(h_, start_, end_, &n, steps.data()));
    if (!withOutputWritersEnabled || writers_.empty()) {
      check(fdm_advance(h_, start_, end_));
      current_time_ = piece_end(n - 1, n);
      piece_steps_ = steps[(size_t)(n - 1)];
      return;
    }
    int64_t done = 0;
    for (int64_t k = 0; k < n; k++) {
      current_time_ = piece_end(k, n);
      piece_steps_ = steps[(size_t)k];
      std::vector<std::pair<OutputWriter*, std::string>> due;
      for (OutputWriter& w : writers_) {
        std::string name;
        if (w.prepare(0, piece_steps_, name))
          due.emplace_back(&w, name);
      }
      if (!due.empty()) {
        check(fdm_advance_pieces(h_, start_, end_, done, k + 1));
        done = k + 1;
        for (auto& d : due)
          if (d.first->write)
            d.first->write(d.second, current_time_);
      }
    }
    if (done < n)
      check(fdm_advance_pieces(h_, start_, end_, done, n));
  }

  /* advanceTimeSpan that returns once the work is enqueued; wait() completes it */
  void advanceTimeSpanAsync()
  {
    initialize();
    if (log_on_)
      grow_stimulation_log(end_ - start_);
    check(fdm_advance_async(h_, start_, end_));
  }
  void wait() { check(fdm_wait(h_)); }
  /* wait() for at most timeoutSeconds: true once the advance is complete, false while it still runs */
  bool waitFor(double timeoutSeconds)
  {
    const int rc = fdm_wait_for(h_, timeoutSeconds);
    if (rc == FDM_ERR_TIMEOUT)
      return false;
    check(rc);
    return true;
  }

  void setTimeSpan(double startTime, double endTime)
  {
    start_ = startTime;
    end_ = endTime;
  }
  double startTime() const { return start_; }
  double endTime() const { return end_; }

  /* Vm, statesForTransfer[1..] and algebraicsForTransfer of every node */
  TransferData data()
  {
    initialize();
    TransferData d;
    const int64_t n = s_.n_nodes();
    int ns = 0, na = 0, np = 0;
    check(fdm_model_info(s_.config.model, &ns, &na, &np, nullptr));
    std::vector<double> st((size_t)ns * n);
    if (n > 0)
      check(fdm_get_states(h_, st.data()));
    d.vm.assign(st.begin(), st.begin() + n);
    for (size_t k = 1; k < s_.states_for_transfer.size(); k++) {
      const int idx = s_.states_for_transfer[k];
      d.states.insert(d.states.end(), st.begin() + (size_t)idx * n, st.begin() + (size_t)(idx + 1) * n);
    }
    if (!s_.algebraics_for_transfer.empty()) {
      d.algebraics.resize(s_.algebraics_for_transfer.size() * (size_t)n);
      check(fdm_get_algebraics(h_, d.algebraics.data()));
    }
    return d;
  }

  /* all states [state][node] */
  std::vector<double> states()
  {
    initialize();
    int ns = 0, na = 0, np = 0;
    check(fdm_model_info(s_.config.model, &ns, &na, &np, nullptr));
    std::vector<double> st((size_t)ns * s_.n_nodes());
    if (!st.empty())
      check(fdm_get_states(h_, st.data()));
    return st;
  }

  void reset()
  {
    if (h_)
      fdm_destroy(h_);
    h_ = nullptr;
  }

  /* Vm at the given nodes after every Strang step from now on (fdm_set_trace; rows count from this call) and,
   * with capacityPerNode > 0, the Strang steps after which their Vm rose above threshold
   * (fdm_set_activation_recording) */
  void traceNodes(const std::vector<int64_t>& nodes, int64_t capacity, double threshold = 0.0,
                  int capacityPerNode = 0)
  {
    initialize();
    trace_nodes_ = nodes;
    act_cap_ = capacityPerNode;
    check(fdm_set_trace(h_, (int)nodes.size(), nodes.data(), capacity));
    if (capacityPerNode > 0)
      check(fdm_set_activation_recording(h_, threshold, capacityPerNode));
  }
  /* the traced Vm, [step * nodes + k] */
  std::vector<double> trace()
  {
    int64_t n = 0;
    check(fdm_get_trace(h_, nullptr, &n));
    std::vector<double> out((size_t)(n * (int64_t)trace_nodes_.size()));
    if (!out.empty())
      check(fdm_get_trace(h_, out.data(), &n));
    return out;
  }
  /* per traced node the Strang steps of its threshold crossings (at most capacityPerNode each) */
  std::vector<std::vector<int>> activationSteps()
  {
    std::vector<int> counts(trace_nodes_.size()), steps(trace_nodes_.size() * (size_t)act_cap_);
    check(fdm_get_activation_steps(h_, counts.data(), steps.data()));
    std::vector<std::vector<int>> out(trace_nodes_.size());
    for (size_t k = 0; k < out.size(); k++)
      for (int j = 0; j < counts[k] && j < act_cap_; j++)
        out[k].push_back(steps[k * (size_t)act_cap_ + (size_t)j]);
    return out;
  }

  /* StimulationLogging: from now on every stimulation begin is recorded (fdm_set_stimulation_log); the capacity
   * grows before each advance to what its span can need */
  void enableStimulationLog()
  {
    initialize();
    log_on_ = true;
    check(fdm_set_stimulation_log(h_, log_bound(s_.end_time - s_.start_time)));
  }

  /* the recorded stimulation begins in time order (fibers numbered by fiber_numbers) */
  std::vector<StimulationLogEntry> stimulationLog()
  {
    initialize();
    int64_t n = 0;
    check(fdm_get_stimulation_log(h_, &n, nullptr, nullptr));
    std::vector<double> t((size_t)(n > 0 ? n : 1));
    std::vector<int> f(t.size());
    check(fdm_get_stimulation_log(h_, &n, t.data(), f.data()));
    std::vector<StimulationLogEntry> out;
    for (int64_t i = 0; i < n && i < (int64_t)t.size(); i++) {
      const int fi = f[(size_t)i];
      out.push_back({t[(size_t)i], s_.motor_unit_no.empty() ? -1 : s_.motor_unit_no[(size_t)fi],
                     s_.fiber_numbers.size() == (size_t)s_.n_fibers() ? s_.fiber_numbers[(size_t)fi] : fi});
    }
    std::sort(out.begin(), out.end(), [](const StimulationLogEntry& a, const StimulationLogEntry& b) {
      return a.time < b.time || (a.time == b.time && a.fiberNo < b.fiberNo);
    });
    return out;
  }

  /* the log file of StimulationLogging::writeLogFile (stimulation_logging.cpp:119-165): sorted by motor unit,
   * fiber and time, a header line and one "<motor unit>;<fiber>;<t1>;<t2>;...;" line per (motor unit, fiber),
   * doubles as a stream writes them; nothing for an empty log */
  void writeStimulationLog(const std::string& filename)
  {
    std::vector<StimulationLogEntry> e = stimulationLog();
    if (e.empty())
      return;
    std::sort(e.begin(), e.end(), [](const StimulationLogEntry& a, const StimulationLogEntry& b) {
      if (a.motorUnitNo != b.motorUnitNo)
        return a.motorUnitNo < b.motorUnitNo;
      if (a.fiberNo != b.fiberNo)
        return a.fiberNo < b.fiberNo;
      return a.time < b.time;
    });
    std::ofstream file(filename);
    if (!file)
      throw Error(FDM_ERR_ARG, "writeStimulationLog: cannot open " + filename);
    file << "# motor unit no; fiber no; stimulation times in ms" << std::endl;
    for (size_t i = 0; i < e.size(); i++) {
      if (i == 0 || e[i].fiberNo != e[i - 1].fiberNo || e[i].motorUnitNo != e[i - 1].motorUnitNo) {
        if (i != 0)
          file << "\n";
        file << e[i].motorUnitNo << ";" << e[i].fiberNo << ";";
      }
      file << e[i].time << ";";
    }
  }

  /* the diffusion's output writers, called after each RepeatedCall piece of advanceTimeSpan(true) */
  void addOutputWriter(OutputWriter w) { writers_.push_back(std::move(w)); }

  /* The reference's callOutputWriter (fast_monodomain_solver_base.tpp:7-24): when timeStepNo is a multiple of
   * callCountIncrement the writers are called as after a RepeatedCall piece, with the end time and split steps
   * of the last piece (0 steps before the first advance: the initial-values call, which always writes);
   * currentTime is not used, as in the reference. */
  void callOutputWriter(int timeStepNo, double currentTime, int callCountIncrement = 1)
  {
    (void)currentTime;
    initialize();
    if (callCountIncrement == 0 || timeStepNo % callCountIncrement != 0)
      return;
    for (OutputWriter& w : writers_) {
      std::string name;
      if (w.prepare(0, piece_steps_, name) && w.write)
        w.write(name, current_time_);
    }
  }

  void saveFiberDataCheckpoint() { check(fdm_checkpoint_save(h_)); }
  void restoreFiberDataCheckpoint() { check(fdm_checkpoint_restore(h_)); }

  fdm_solver* handle() { return h_; }
  const FiberSettings& settings() const { return s_; }

 private:
  void check(int rc)
  {
    if (rc != FDM_OK)
      throw Error(rc, fdm_last_error(h_));
  }

  /* CellmlAdapter::initializeToEquilibriumValues (03_cellml_adapter.tpp:445-515) for the first node's states
   * and parameters; every node starts from the result */
  void initialize_to_equilibrium()
  {
    int ns = 0, na = 0, np = 0;
    check(fdm_model_info(s_.config.model, &ns, &na, &np, nullptr));
    const int64_t n = s_.n_nodes();
    std::vector<double> y((size_t)ns), p((size_t)(np > 0 ? np : 1), 0.0);
    if (s_.states.empty()) {
      check(fdm_model_info(s_.config.model, &ns, &na, &np, y.data()));
    } else {
      for (int k = 0; k < ns; k++)
        y[(size_t)k] = s_.states[(size_t)k * (size_t)n];
    }
    if (!s_.parameters.empty())
      for (int q = 0; q < np; q++)
        p[(size_t)q] = s_.parameters[(size_t)q * (size_t)n];
    else if (np > 0)
      check(fdm_model_parameter_defaults(s_.config.model, p.data()));
    const int rc = fdm_model_equilibrium(s_.config.model, s_.config.device, s_.config.approximate_exponential_function,
                                         p.data(), s_.equilibrium_dt, y.data(), &equilibrium_iterations_, nullptr,
                                         nullptr);
    if (rc != FDM_OK)
      throw Error(rc, fdm_last_error(nullptr));
    s_.states.assign((size_t)ns * (size_t)n, 0.0);
    for (int k = 0; k < ns; k++)
      for (int64_t i = 0; i < n; i++)
        s_.states[(size_t)k * (size_t)n + (size_t)i] = y[(size_t)k];
    equilibrium_done_ = true;
  }

  /* stimulation begins a span can hold: a fiber's machine checks at most once per 1/(f (1 + |jitter|)) */
  int64_t log_bound(double span) const
  {
    int64_t b = 16;
    for (int f = 0; f < s_.n_fibers(); f++) {
      double jmax = 0.0;
      for (int k = 0; k < s_.n_jitter; k++)
        jmax = std::max(jmax, std::fabs(s_.jitter[(size_t)f * (size_t)s_.n_jitter + (size_t)k]));
      b += (int64_t)std::ceil(std::max(span, 0.0) * s_.call_frequency[(size_t)f] * (1.0 + jmax)) + 2;
    }
    return b;
  }

  void grow_stimulation_log(double span)
  {
    int64_t n = 0;
    check(fdm_get_stimulation_log(h_, &n, nullptr, nullptr));
    check(fdm_set_stimulation_log(h_, n + log_bound(span)));
  }

  /* end of RepeatedCall piece k of n (the Strang span's end time: start + k/n*span + span/n) */
  double piece_end(int64_t k, int64_t n) const
  {
    const double span = end_ - start_;
    const double t = k == 0 ? start_ : start_ + (double)k / (double)n * span;
    return t + span / (double)n;
  }

  FiberSettings s_;
  fdm_solver* h_ = nullptr;
  double start_ = 0.0, end_ = 0.0;
  std::vector<OutputWriter> writers_;
  double current_time_ = 0.0;  // the reference's currentTime_: end of the last RepeatedCall piece
  int piece_steps_ = 0;        // its number of split steps (nTimeStepsSplitting_)
  bool log_on_ = false;
  std::vector<int64_t> trace_nodes_;
  int act_cap_ = 0;
  bool equilibrium_done_ = false;
  int64_t equilibrium_iterations_ = 0;
};

}  // namespace fdm

#endif /* FDM_B200_HPP */
