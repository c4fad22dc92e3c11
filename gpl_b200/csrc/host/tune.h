// The engine's autotuner: picks, where it runs, the fastest of a launch group's forms that
// give the same results bit for bit (the SpMV's three row layouts, the scatter's shared-tile
// and straight-to-HBM forms, the small nets' three WA kernels). Which form wins depends on
// the data (row lengths, how far a block's cells spread, the degree mix) and changes as the
// loop moves cells, so each Tuner times its candidates in place with CUDA events on the
// stream they run on: every candidate in turn for a few uses, then the fastest by its median
// time, and the probe again every `period` uses. A use is bracketed by start() and stop();
// finish() is called once the stream has synchronised (the trial's read-back, the solver's
// batch read), reads the use's time and counts it or, for a use that did less work than the
// others (a solver batch that ended part-way), drops it. A probe that keeps the form in use
// doubles the period to the next (up to 16 times `period`); one that changes it starts over.
//
// An environment variable can fix the form instead (its accepted values name the candidates
// in order): the forms give the same results, so it changes only the speed.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace gpl {

class Tuner {
 public:
  // `names` names the candidates (their count is the candidate count); `env`, when set in the
  // environment to one of the names, fixes that candidate.
  Tuner(std::string what, std::vector<std::string> names, const char *env, int probe = 3, int period = 256);
  ~Tuner();
  Tuner(const Tuner &) = delete;
  Tuner &operator=(const Tuner &) = delete;

  // The candidate this use runs, with the start event recorded on `s` when the use is timed.
  int start(cudaStream_t s);
  void stop(cudaStream_t s);
  // After the stream has synchronised: the use's time counted (or dropped), the choice updated.
  void finish(bool count = true);
  int best() const { return best_; }
  bool fixed() const { return fixed_ >= 0; }
  int64_t probes() const { return probes_; }
  // "what: name (a / b / c us)", the candidates' last median times.
  std::string report() const;

 private:
  std::string what_;
  std::vector<std::string> names_;
  int n_ = 0, probe_ = 3, base_period_ = 256, period_ = 256;
  int fixed_ = -1;
  int best_ = 0;
  int cur_ = 0;              // the candidate of the use in flight
  bool timed_ = false;       // the use in flight is a probe's
  bool in_flight_ = false;
  bool probing_ = true;
  int probe_pos_ = 0;        // uses of the probe launched so far
  int64_t since_ = 0;        // uses since the last probe ended
  int64_t probes_ = 0;
  std::vector<std::vector<float>> samples_;
  std::vector<float> median_;
  cudaEvent_t ev_[2] = {nullptr, nullptr};
  void decide();
};

}  // namespace gpl
