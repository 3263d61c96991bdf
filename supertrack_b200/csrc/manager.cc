// Reference-shaped C++ classes (supertrack.h) and the macro-level C ABI entry points.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <sstream>

#include "supertrack.h"

namespace st {

namespace {
int ZShiftFromString(const std::string& s) {
  std::string v = s;
  for (auto& ch : v) ch = (char)std::tolower((unsigned char)ch);
  if (v == "minus" || v == "-") return ST_ZSHIFT_MINUS;
  if (v == "none" || v == "0" || v == "off") return ST_ZSHIFT_NONE;
  return ST_ZSHIFT_PLUS;
}

int HistTypeFromString(const std::string& s) {
  if (s == "lin") return ST_HIST_LIN;
  if (s == "log") return ST_HIST_LOG;
  return -1;
}
}  // namespace

// ---------------------------------------------------------------------------------------------
SphericalGeometry::SphericalGeometry(double hl, double d) {
  st_geometry g;
  valid = st_geometry_make(hl, d, &g) == ST_OK;
  if (valid) {
    scoringRegionLength = g.scoring_region_length;
    scoringRegionHalfLength = g.scoring_region_half_length;
    greatestSphereOffset = g.greatest_sphere_offset;
    numSpheresLinear = g.num_spheres_linear;
    sphereDiameter = g.sphere_diameter;
    sphereRadius = g.sphere_radius;
  }
}

SphericalGeometry::SphericalGeometry(const INIReader& r)
    : SphericalGeometry(r.GetReal("VoxelConstrainedSphere", "ScoringRegionHalfLength", 0),
                        r.GetReal("VoxelConstrainedSphere", "ScoringSphereDiameter", 0)) {}

// ---------------------------------------------------------------------------------------------
bool Track::AllocateAndLoadTrack(const ThreadTask& task) {
  const int64_t n = task.exitPoint - task.entryPoint;
  if (n < 0) return false;
  x.resize(n); y.resize(n); z.resize(n); edep.resize(n);
  return ReadTrackDeposits(task.fileName, task.entryPoint, task.exitPoint, x.data(), y.data(),
                           z.data(), edep.data());
}

void Track::Free() {
  std::vector<double>().swap(x);
  std::vector<double>().swap(y);
  std::vector<double>().swap(z);
  std::vector<double>().swap(edep);
}

// ---------------------------------------------------------------------------------------------
SimulationMethodFactory& SimulationMethodFactory::GetInstance() {
  static SimulationMethodFactory singleton;
  return singleton;
}

void SimulationMethodFactory::AddSimulationMethod(const std::string& name, SimulationMethodCtor ctor) {
  for (auto& p : _nameConstructorPairs)
    if (p.first == name) { p.second = ctor; return; }
  _nameConstructorPairs.emplace_back(name, ctor);
}

SimulationMethod* SimulationMethodFactory::Construct(const INIReader& reader) const {
  const std::string name = reader.Get("Simulation", "Method", "");
  for (const auto& p : _nameConstructorPairs)
    if (p.first == name) return p.second(reader);
  return nullptr;
}

// ---------------------------------------------------------------------------------------------
VoxelConstrainedSphereMethod::VoxelConstrainedSphereMethod(const INIReader& r)
    : SimulationMethod(r), _sphericalGeometry(r) {
  ParseInput();
}

SimulationMethod* VoxelConstrainedSphereMethod::Construct(const INIReader& r) {
  return new VoxelConstrainedSphereMethod(r);
}

void VoxelConstrainedSphereMethod::ParseInput() {
  _randomShifts = _macroReader.GetBoolean("VoxelConstrainedSphere", "ShiftTrack", true);
  _zshift = ZShiftFromString(_macroReader.Get("VoxelConstrainedSphere", "ZOriginShift", "plus"));
}

void VoxelConstrainedSphereMethod::AllocateTrackProcess(Track&, ThreadTask task) {
  _taskSeed = task.randomSeed;
  _oversampleIterationNumber = 0;
}

void VoxelConstrainedSphereMethod::ProcessTrack(Track& track, VolumeEdepPair& pair) {
  pair.producer = this;
  pair.track = &track;
  pair.pending += 1;
  ++_oversampleIterationNumber;
}

void VoxelConstrainedSphereMethod::FreeTrackProcess() { _oversampleIterationNumber = 0; }

st_job_desc VoxelConstrainedSphereMethod::JobFor(uint32_t n_oversamples) const {
  st_job_desc d;
  std::memset(&d, 0, sizeof(d));
  d.half_length = _macroReader.GetReal("VoxelConstrainedSphere", "ScoringRegionHalfLength", 0);
  d.sphere_diameter = _macroReader.GetReal("VoxelConstrainedSphere", "ScoringSphereDiameter", 0);
  d.zshift = _zshift;
  d.shift_track = _randomShifts ? 1 : 0;
  d.n_oversamples = n_oversamples;
  d.seed = (uint64_t)_taskSeed;
  d.track_id = 0;
  d.hist_id = -1;
  return d;
}

// ---------------------------------------------------------------------------------------------
Histogram::Histogram(int nbins, float lo, float hi, const std::string& type, st_ctx* ctx) : _ctx(ctx) {
  const int t = HistTypeFromString(type);
  int32_t id = -1;
  _status = t < 0 ? ST_ERR_BAD_HISTOGRAM : st_hist_create(ctx, t, nbins, lo, hi, &id);
  if (_status == ST_OK) {
    _id = id;
    _nbins = nbins;
    _edges.resize((size_t)nbins + 1);
    st_hist_edges_of(ctx, id, _edges.data());
  }
}

Histogram::Histogram(const INIReader& r, st_ctx* ctx)
    : Histogram((int)r.GetInteger("Histogram", "NBins", 0), r.GetFloat("Histogram", "BinLower", 0),
                r.GetFloat("Histogram", "BinUpper", 0), r.Get("Histogram", "Type", ""), ctx) {}

void Histogram::AllocateTrackProcess(VolumeEdepPair& pair) {
  _pending = &pair;
  _consumed = 0;
}

void Histogram::SortReduceAndAddToHistogram(VolumeEdepPair& pair) {
  _pending = &pair;
  _consumed = pair.pending;
}

void Histogram::FreeTrackProcess() {
  if (_status != ST_OK || !_pending || !_pending->producer || !_pending->track || _consumed == 0) {
    _pending = nullptr;
    return;
  }
  const Track& t = *_pending->track;
  st_track_view v;
  std::memset(&v, 0, sizeof(v));
  v.x = t.x.data(); v.y = t.y.data(); v.z = t.z.data(); v.edep = t.edep.data();
  v.n = t.Size();
  v.on_device = 0;
  st_job_desc d = _pending->producer->JobFor(_consumed);
  d.hist_id = _id;
  int32_t job = -1;
  st_status s = st_job_submit(_ctx, &v, &d, &job);
  if (s == ST_OK) s = st_run(_ctx, ST_RUN_PLAIN);
  if (s == ST_OK) s = st_jobs_clear(_ctx);
  if (s != ST_OK) _status = s;
  _pending->pending = 0;
  _pending = nullptr;
  _consumed = 0;
}

bool Histogram::GetCPUHistogram(std::vector<int64_t>* counts, std::vector<double>* yfy) const {
  if (_status != ST_OK && _id < 0) return false;
  if (counts) counts->assign((size_t)_nbins, 0);
  if (yfy) yfy->assign((size_t)_nbins, 0.0);
  return st_hist_read(_ctx, _id, counts ? counts->data() : nullptr, yfy ? yfy->data() : nullptr) == ST_OK;
}

// ---------------------------------------------------------------------------------------------
SuperTrackManager& SuperTrackManager::GetInstance() {
  static SuperTrackManager singleton;
  return singleton;
}

void SuperTrackManager::AddSimulationMethod(const std::string& name, SimulationMethodCtor ctor) {
  SimulationMethodFactory::GetInstance().AddSimulationMethod(name, ctor);
}

void SuperTrackManager::Reset() {
  _threadAllocations.clear();
  _counts.clear();
  _yfy.clear();
  _edges.clear();
  _deposits = 0;
  _initialized = false;
  _runStatus = ST_OK;
}

std::string SuperTrackManager::Initialize(const std::string& iniPath, int device) {
  Reset();
  _reader = INIReader(iniPath);
  if (_reader.ParseError() == -1) return "Cannot open macro file: " + iniPath;
  if (_reader.ParseError() > 0) return "Macro parse error on line " + std::to_string(_reader.ParseError());
  std::string e = ReadRunConfig(_reader, &_cfg);
  if (!e.empty()) return e;
  e = ReturnThreadAllocations(_cfg, &_threadAllocations);
  if (!e.empty()) return e;
  _device = device;
  _initialized = true;
  return "";
}

std::string SuperTrackManager::Run(bool writeOutput) {
  if (!_initialized) return "Can not start run without initializing manager.";
  _runStatus = ST_OK;
  std::unique_ptr<SimulationMethod> method(SimulationMethodFactory::GetInstance().Construct(_reader));
  if (!method)
    return "No simulation method matching name: " + _reader.Get("Simulation", "Method", "") + " found.";
  st_ctx* ctx = nullptr;
  st_status s = st_ctx_create(_device, nullptr, &ctx);
  if (s != ST_OK) {
    _runStatus = s;
    return std::string("GPU context: ") + st_status_string(s);
  }
  std::string err;
  {
    Histogram histogram(_reader, ctx);
    if (histogram.Status() != ST_OK) {
      err = "Unknown or invalid histogram: " + _reader.Get("Histogram", "Type", "") +
            " (available types are lin and log; bounds must give increasing edges)";
    }
    // Tracks are loaded into host memory and submitted in groups of at most kGroupDeposits
    // deposits; each group runs as one batched launch.
    const int64_t kGroupDeposits = (int64_t)1 << 27;
    std::vector<std::unique_ptr<Track>> group;
    int64_t group_deposits = 0;
    auto flush = [&]() -> bool {
      if (group.empty()) return true;
      st_status rs = st_run(ctx, ST_RUN_BATCHED);
      if (rs == ST_OK) rs = st_jobs_clear(ctx);
      group.clear();
      group_deposits = 0;
      if (rs != ST_OK) {
        char buf[256];
        st_ctx_last_error(ctx, buf, sizeof(buf));
        err = std::string("GPU run failed: ") + st_status_string(rs) + " " + buf;
        _runStatus = rs;
        return false;
      }
      return true;
    };
    for (auto& alloc : _threadAllocations) {
      if (!err.empty()) break;
      for (auto& task : alloc.tasks) {
        std::unique_ptr<Track> track(new Track());
        if (!track->AllocateAndLoadTrack(task)) { err = "Cannot read track from " + task.fileName; break; }
        method->AllocateTrackProcess(*track, task);
        st_job_desc d = method->JobFor((uint32_t)task.nOversamples);
        d.hist_id = histogram.Id();
        st_track_view v;
        std::memset(&v, 0, sizeof(v));
        v.x = track->x.data(); v.y = track->y.data(); v.z = track->z.data(); v.edep = track->edep.data();
        v.n = track->Size();
        s = st_job_submit(ctx, &v, &d, nullptr);
        if (s != ST_OK) {
          err = std::string("Job rejected: ") + st_status_string(s);
          _runStatus = s;
          break;
        }
        method->FreeTrackProcess();
        _deposits += track->Size();
        group_deposits += track->Size();
        group.push_back(std::move(track));
        if (group_deposits >= kGroupDeposits && !flush()) break;
      }
    }
    if (err.empty()) flush();
    if (err.empty()) {
      histogram.GetCPUHistogram(&_counts, &_yfy);
      _edges = histogram.Edges();
    }
  }
  st_ctx_destroy(ctx);
  if (!err.empty()) return err;
  if (writeOutput) return EndOfRun();
  return "";
}

std::string SuperTrackManager::EndOfRun() {
  const std::string folder = _reader.Get("Output", "Path", "");
  const std::string prefix = _reader.Get("Output", "NamePrefix", "");
  const long long seed = _threadAllocations.empty() ? _cfg.randomSeed : _threadAllocations[0].randomSeed;
  std::stringstream base;
  base << folder << prefix << seed;
  int64_t ntracks = 0;
  for (auto& a : _threadAllocations) ntracks += (int64_t)a.tasks.size();
  {
    std::ofstream csv(base.str() + ".csv");
    if (!csv) return "Cannot write output " + base.str() + ".csv";
    csv.precision(17);
    csv << "bin_lower,bin_upper,counts,yfy\n";
    for (size_t i = 0; i < _counts.size(); ++i)
      csv << _edges[i] << "," << _edges[i + 1] << "," << _counts[i] << "," << _yfy[i] << "\n";
  }
  {
    std::ofstream js(base.str() + ".json");
    if (!js) return "Cannot write output " + base.str() + ".json";
    js << "{\"title\": \"N(y)\", \"Number of Tracks\": " << ntracks
       << ", \"Number of Oversamples\": " << _cfg.oversamples
       << ", \"Effective Number of Tracks\": " << ntracks * _cfg.oversamples
       << ", \"random_seed\": " << seed << ", \"deposits\": " << _deposits
       << ", \"nbins\": " << _counts.size() << "}\n";
  }
  return "";
}

}  // namespace st

// =============================================================================================
// Macro-level C ABI
// =============================================================================================
struct st_ini {
  st::INIReader r;
};

extern "C" {

st_status st_run_macro(const char* ini_path, int32_t device, int32_t write_output, int64_t* counts,
                       double* yfy, int32_t nbins_cap, st_run_info* info, char* err, size_t err_len) {
  auto fail = [&](st_status s, const std::string& m) {
    if (err && err_len) std::snprintf(err, err_len, "%s", m.c_str());
    return s;
  };
  if (!ini_path) return fail(ST_ERR_INVALID_ARGUMENT, "null macro path");
  auto& mgr = st::SuperTrackManager::GetInstance();
  mgr.AddSimulationMethod("VoxelConstrainedSphere", &st::VoxelConstrainedSphereMethod::Construct);
  std::string e = mgr.Initialize(ini_path, device);
  if (!e.empty()) return fail(ST_ERR_CONFIG, e);
  e = mgr.Run(write_output != 0);
  if (!e.empty()) {
    const st_status g = mgr.RunStatus();
    return fail(g != ST_OK ? g : ST_ERR_CONFIG, e);
  }
  const auto& c = mgr.GetOutputCounts();
  const auto& y = mgr.GetOutputYFY();
  if ((size_t)nbins_cap < c.size() && (counts || yfy)) return fail(ST_ERR_CAPACITY, "nbins_cap too small");
  if (counts) std::memcpy(counts, c.data(), c.size() * 8);
  if (yfy) std::memcpy(yfy, y.data(), y.size() * 8);
  if (info) {
    std::memset(info, 0, sizeof(*info));
    int64_t nt = 0;
    for (auto& a : mgr.Allocations()) nt += (int64_t)a.tasks.size();
    st::INIReader r(ini_path);
    info->n_tracks = nt;
    info->n_oversamples = r.GetInteger("Run", "Oversamples", 1);
    info->n_effective = nt * info->n_oversamples;
    info->random_seed = mgr.Allocations().empty() ? 0 : mgr.Allocations()[0].randomSeed;
    info->deposits = mgr.Deposits();
    info->nbins = (int32_t)c.size();
  }
  return ST_OK;
}

st_status st_macro_tasks(const char* ini_path, st_task* tasks, int64_t cap, int64_t* n_out,
                         char* err, size_t err_len) {
  auto fail = [&](st_status s, const std::string& m) {
    if (err && err_len) std::snprintf(err, err_len, "%s", m.c_str());
    return s;
  };
  if (!ini_path || !n_out) return fail(ST_ERR_INVALID_ARGUMENT, "null argument");
  st::INIReader r(ini_path);
  if (r.ParseError() == -1) return fail(ST_ERR_IO, std::string("cannot open ") + ini_path);
  st::RunConfig cfg;
  std::string e = st::ReadRunConfig(r, &cfg);
  if (!e.empty()) return fail(ST_ERR_CONFIG, e);
  std::vector<st::ThreadAllocation> allocs;
  e = st::ReturnThreadAllocations(cfg, &allocs);
  if (!e.empty()) return fail(ST_ERR_CONFIG, e);
  int64_t n = 0;
  for (auto& a : allocs) n += (int64_t)a.tasks.size();
  *n_out = n;
  if (!tasks) return ST_OK;
  if (n > cap) return fail(ST_ERR_CAPACITY, "task buffer too small");
  // file ordinal: position of the task's file in the sorted folder listing (1-based)
  std::vector<std::string> files;
  int64_t k = 0;
  for (auto& a : allocs) {
    for (auto& t : a.tasks) {
      int32_t ord = 0;
      for (size_t f = 0; f < files.size(); ++f)
        if (files[f] == t.fileName) ord = (int32_t)f + 1;
      if (!ord) { files.push_back(t.fileName); ord = (int32_t)files.size(); }
      tasks[k].entry = t.entryPoint;
      tasks[k].exit = t.exitPoint;
      tasks[k].seed = t.randomSeed;
      tasks[k].thread_id = t.threadID;
      tasks[k].file_ordinal = ord + (int32_t)(cfg.firstFile > 0 ? cfg.firstFile - 1 : 0);
      tasks[k].n_oversamples = t.nOversamples;
      tasks[k].track_in_file = t.trackInFile;
      ++k;
    }
  }
  return ST_OK;
}

st_status st_track_file_write(const char* path, uint64_t n_tracks, const uint64_t* index,
                              uint64_t n_deposits, const double* x, const double* y,
                              const double* z, const double* edep) {
  if (!path || (n_tracks && !index) || (n_deposits && (!x || !y || !z || !edep)))
    return ST_ERR_INVALID_ARGUMENT;
  uint64_t prev = 0;
  for (uint64_t i = 0; i < n_tracks; ++i) {
    if (index[i] < prev || index[i] > n_deposits) return ST_ERR_INVALID_ARGUMENT;
    prev = index[i];
  }
  return st::WriteTrackFile(path, n_tracks, index, n_deposits, x, y, z, edep) ? ST_OK : ST_ERR_IO;
}

st_status st_ini_open(const char* path, st_ini** out, int32_t* parse_error) {
  if (!path || !out) return ST_ERR_INVALID_ARGUMENT;
  st_ini* h = new st_ini{st::INIReader(path)};
  if (parse_error) *parse_error = h->r.ParseError();
  *out = h;
  return h->r.ParseError() == -1 ? ST_ERR_IO : ST_OK;
}

st_status st_ini_from_string(const char* text, st_ini** out, int32_t* parse_error) {
  if (!text || !out) return ST_ERR_INVALID_ARGUMENT;
  st_ini* h = new st_ini{st::INIReader::FromString(text)};
  if (parse_error) *parse_error = h->r.ParseError();
  *out = h;
  return ST_OK;
}

void st_ini_close(st_ini* ini) { delete ini; }

st_status st_ini_get(const st_ini* ini, const char* section, const char* name,
                     const char* default_value, char* buf, size_t len) {
  if (!ini || !section || !name || !buf || !len) return ST_ERR_INVALID_ARGUMENT;
  const std::string v = ini->r.Get(section, name, default_value ? default_value : "");
  if (v.size() + 1 > len) return ST_ERR_CAPACITY;
  std::memcpy(buf, v.c_str(), v.size() + 1);
  return ST_OK;
}

long st_ini_get_integer(const st_ini* ini, const char* s, const char* n, long d) {
  return ini ? ini->r.GetInteger(s, n, d) : d;
}
double st_ini_get_real(const st_ini* ini, const char* s, const char* n, double d) {
  return ini ? ini->r.GetReal(s, n, d) : d;
}
float st_ini_get_float(const st_ini* ini, const char* s, const char* n, float d) {
  return ini ? ini->r.GetFloat(s, n, d) : d;
}
int32_t st_ini_get_boolean(const st_ini* ini, const char* s, const char* n, int32_t d) {
  return ini ? (ini->r.GetBoolean(s, n, d != 0) ? 1 : 0) : d;
}

st_status st_spectrum_bin_log_x(int32_t nbins, double from_log10, double to_log10, double* edges) {
  if (nbins < 1 || !edges) return ST_ERR_INVALID_ARGUMENT;
  st::CPUHistogramUtils::BinLogX(nbins, from_log10, to_log10, edges);
  return ST_OK;
}

st_status st_spectrum_pmf_to_pdf(int32_t nbins, const double* edges, double* contents) {
  if (nbins < 1 || !edges || !contents) return ST_ERR_INVALID_ARGUMENT;
  st::CPUHistogramUtils::PMF_to_PDF(nbins, edges, contents);
  return ST_OK;
}

st_status st_spectrum_prepare_for_semilog(int32_t nbins, const double* edges, double* contents) {
  if (nbins < 1 || !edges || !contents) return ST_ERR_INVALID_ARGUMENT;
  st::CPUHistogramUtils::Prepare_for_Semilog(nbins, edges, contents);
  return ST_OK;
}

}  // extern "C"
