// C++ surface of the reference kept for drop-in use: SimulationMethod and its factory,
// VoxelConstrainedSphereMethod, SphericalGeometry, Track, VolumeEdepPair, Histogram and the
// SuperTrackManager run loop. The classes keep the reference's names, call protocol and argument
// meaning; underneath, every track's oversamples run as one job of the fused sm_100a kernel
// through the C ABI (include/supertrack_b200.h).
//
// Differences from the reference that a caller can observe:
//   * errors are reported (return codes / Status()) instead of abort();
//   * the track is never modified (the reference shifts track.z in place,
//     VoxelConstrainedSphereMethod.cu:45);
//   * ProcessTrack/SortReduceAndAddToHistogram only record the oversamples; the fused kernel
//     runs when the histogram's FreeTrackProcess closes the track;
//   * the histogram is an int64 f(y) plus a float64 y*f(y) spectrum instead of a ROOT TH1D.
#pragma once
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/supertrack_b200.h"
#include "host_model.h"

namespace st {

// SphericalGeometry (SphericalGeometry.cuh:8-23) constructed from (HL, d) or the macro.
struct ST_CXX_API SphericalGeometry {
  SphericalGeometry(double scoring_region_half_length, double sphere_diameter);
  explicit SphericalGeometry(const INIReader& reader);
  double scoringRegionLength = 0;
  double scoringRegionHalfLength = 0;
  double greatestSphereOffset = 0;
  int numSpheresLinear = 0;
  double sphereDiameter = 0;
  double sphereRadius = 0;
  bool valid = false;
};

// Host-resident SoA track (Track.cuh:7-22); AllocateAndLoadTrack reads a task's deposits from
// its track file.
class ST_CXX_API Track {
 public:
  bool AllocateAndLoadTrack(const ThreadTask& task);
  void Free();
  std::vector<double> x, y, z, edep;
  int64_t Size() const { return (int64_t)x.size(); }
};

class SimulationMethod;

// The per-track hand-off between the simulation method and the histogram (VolumeEdepPair.cuh).
// It records which oversamples of which track are pending instead of holding per-hit pairs.
class ST_CXX_API VolumeEdepPair {
 public:
  void Allocate(uint64_t /*numInputElements*/) { pending = 0; }
  void Free() { pending = 0; }
  SimulationMethod* producer = nullptr;
  const Track* track = nullptr;
  uint32_t pending = 0;
};

class ST_CXX_API SimulationMethod {
 public:
  explicit SimulationMethod(const INIReader& macroReader) : _macroReader(macroReader) {}
  virtual ~SimulationMethod() = default;
  virtual void ParseInput() = 0;
  virtual void AllocateTrackProcess(Track& track, ThreadTask task) = 0;
  virtual void ProcessTrack(Track& track, VolumeEdepPair& edepsInTarget) = 0;
  virtual void FreeTrackProcess() = 0;
  virtual void Free() = 0;
  // The job description of the current track (geometry, shifts, seed, oversamples).
  virtual st_job_desc JobFor(uint32_t n_oversamples) const = 0;

 protected:
  INIReader _macroReader;
};

using SimulationMethodCtor = SimulationMethod* (*)(const INIReader&);

// Name -> constructor registry (SimulationMethodFactory.hh:12-37). Construct returns nullptr when
// no registered name matches [Simulation] Method.
class ST_CXX_API SimulationMethodFactory {
 public:
  static SimulationMethodFactory& GetInstance();
  void AddSimulationMethod(const std::string& name, SimulationMethodCtor ctor);
  SimulationMethod* Construct(const INIReader& reader) const;
  void Clear() { _nameConstructorPairs.clear(); }

 private:
  SimulationMethodFactory() = default;
  std::vector<std::pair<std::string, SimulationMethodCtor>> _nameConstructorPairs;
};

// VoxelConstrainedSphereMethod (VoxelConstrainedSphereMethod.hh). Reads
// [VoxelConstrainedSphere] ScoringRegionHalfLength, ScoringSphereDiameter, ShiftTrack and the
// added ZOriginShift = plus|minus|none (default plus, the reference's +HL'). The
// SuggestedCudaBlocks/Threads keys are accepted and ignored: the fused kernel picks its own
// launch shape.
class ST_CXX_API VoxelConstrainedSphereMethod : public SimulationMethod {
 public:
  explicit VoxelConstrainedSphereMethod(const INIReader& macroReader);
  static SimulationMethod* Construct(const INIReader& macroReader);
  void ParseInput() override;
  void AllocateTrackProcess(Track& track, ThreadTask task) override;
  void ProcessTrack(Track& track, VolumeEdepPair& edepsInTarget) override;
  void FreeTrackProcess() override;
  void Free() override {}
  st_job_desc JobFor(uint32_t n_oversamples) const override;
  const SphericalGeometry& Geometry() const { return _sphericalGeometry; }
  bool ShiftTrack() const { return _randomShifts; }
  int ZShiftMode() const { return _zshift; }

 private:
  SphericalGeometry _sphericalGeometry;
  bool _randomShifts = true;
  int _zshift = ST_ZSHIFT_PLUS;
  int64_t _taskSeed = 0;
  int _oversampleIterationNumber = 0;
};

// Histogram (Histogram.cuh:15-72) over a shared GPU context. f(y) counts are exact int64 sums;
// y*f(y) is a float64 sum per bin.
class ST_CXX_API Histogram {
 public:
  Histogram(int nbins, float binLower, float binUpper, const std::string& type, st_ctx* ctx);
  Histogram(const INIReader& reader, st_ctx* ctx);
  Histogram(const Histogram&) = delete;
  void operator=(const Histogram&) = delete;

  void AllocateTrackProcess(VolumeEdepPair& targetEdeps);
  void SortReduceAndAddToHistogram(VolumeEdepPair& targetEdeps);
  void FreeTrackProcess();

  // Copies the device spectrum to host vectors.
  bool GetCPUHistogram(std::vector<int64_t>* counts, std::vector<double>* yfy) const;
  const std::vector<double>& Edges() const { return _edges; }
  int NBins() const { return _nbins; }
  int Id() const { return _id; }
  st_status Status() const { return _status; }

 private:
  st_ctx* _ctx;
  int _id = -1;
  int _nbins = 0;
  std::vector<double> _edges;
  VolumeEdepPair* _pending = nullptr;
  uint32_t _consumed = 0;
  st_status _status = ST_OK;
};

// SuperTrackManager (SuperTrackManager.hh). Run() loads every task's track and runs all of them
// as one batched launch per memory-bounded group of tracks, summing into one spectrum.
class ST_CXX_API SuperTrackManager {
 public:
  static SuperTrackManager& GetInstance();
  void AddSimulationMethod(const std::string& name, SimulationMethodCtor ctor);
  // Returns an empty string on success or the error.
  std::string Initialize(const std::string& iniPath, int device = 0);
  std::string Run(bool writeOutput = true);
  const std::vector<int64_t>& GetOutputCounts() const { return _counts; }
  const std::vector<double>& GetOutputYFY() const { return _yfy; }
  const std::vector<double>& GetOutputEdges() const { return _edges; }
  const std::vector<ThreadAllocation>& Allocations() const { return _threadAllocations; }
  int64_t Deposits() const { return _deposits; }
  // Status of the library call (context, job submit, GPU run) that stopped the last Run; ST_OK
  // when none did, including when Run stopped on the macro or the track files instead.
  st_status RunStatus() const { return _runStatus; }
  void Reset();

 private:
  SuperTrackManager() = default;
  std::string EndOfRun();
  INIReader _reader;
  RunConfig _cfg;
  std::vector<ThreadAllocation> _threadAllocations;
  std::vector<int64_t> _counts;
  std::vector<double> _yfy;
  std::vector<double> _edges;
  int64_t _deposits = 0;
  int _device = 0;
  bool _initialized = false;
  st_status _runStatus = ST_OK;
};

}  // namespace st
