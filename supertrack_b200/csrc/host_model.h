// Host-side model of the reference surface for the VoxelConstrainedSphere path: the .ini
// reader, histogram bin edges, the task/seed allocation over a track folder and the track file
// format that replaces the ROOT "Tracks"/"Track index" trees.
#pragma once
#include <stdint.h>
#include <map>
#include <set>
#include <string>
#include <vector>

// The library builds with hidden visibility; the C ABI and the C++ surface marked ST_CXX_API (this
// header and supertrack.h) are what it exports, so C++ callers can link the classes directly.
#if defined(__GNUC__)
#define ST_CXX_API __attribute__((visibility("default")))
#else
#define ST_CXX_API
#endif

namespace st {

// ---------------------------------------------------------------------------------------------
// INI reader with the semantics of the inih INIReader the reference uses
// (extern/inih/INIReader.h): case-insensitive section/name lookup (:442-448), ';' and '#'
// full-line comments, ';' inline comments only after whitespace (:145-149), '=' or ':'
// separators, indented continuation lines appended with "\n" (:450-460), numbers parsed with
// strtol(...,0)/strtod/strtof and the default returned when nothing parses (:401-427), booleans
// true/yes/on/1 and false/no/off/0 (:429-440). ParseError() is 0, the first bad line, or -1 when
// the file cannot be opened.
// ---------------------------------------------------------------------------------------------
class ST_CXX_API INIReader {
 public:
  explicit INIReader(const std::string& filename);
  static INIReader FromString(const std::string& text);
  INIReader() = default;

  int ParseError() const { return _error; }
  const std::set<std::string>& Sections() const { return _sections; }
  std::string Get(const std::string& section, const std::string& name,
                  const std::string& default_value) const;
  long GetInteger(const std::string& section, const std::string& name, long default_value) const;
  double GetReal(const std::string& section, const std::string& name, double default_value) const;
  float GetFloat(const std::string& section, const std::string& name, float default_value) const;
  bool GetBoolean(const std::string& section, const std::string& name, bool default_value) const;
  bool Has(const std::string& section, const std::string& name) const;

 private:
  void ParseText(const std::string& text);
  static std::string MakeKey(const std::string& section, const std::string& name);
  int _error = 0;
  std::map<std::string, std::string> _values;
  std::set<std::string> _sections;
};

// ---------------------------------------------------------------------------------------------
// Bin edges (utils.cc:8-31 as called from Histogram.cu:53-72). Bounds arrive as float (the
// reference reads them with GetFloat); the linear width is a float expression; the log bounds
// are log10 values stored as float. Returns false for an unknown type, nbins < 1, or edges that
// are not finite and strictly increasing (for example a log histogram with a bound <= 0).
// ---------------------------------------------------------------------------------------------
ST_CXX_API void LinSpace(float bottom, float top, int nbins, double* bins);
ST_CXX_API void LogSpace(float bottom, float top, int nbins, double* bins);
ST_CXX_API bool MakeEdges(int type, int nbins, float lower, float upper, std::vector<double>* edges);

// ---------------------------------------------------------------------------------------------
// Spectrum post-processing (CPUHistogramUtils, utils.cc:37-117). The reference applies these to
// a ROOT TH1 built with the bin edges, whose contents are indexed like ROOT's: 0 is the
// underflow bin, 1..nbins the bins, nbins+1 the overflow bin. `contents` has that layout here
// (nbins + 2 values). The reference's loops run over indices 0..nbins-1, so they touch the
// underflow bin (with ROOT's equidistant low edge below the axis) and leave the last bin alone;
// its normalisation sum is a float. Both are kept, so the outputs equal the reference's.
// ---------------------------------------------------------------------------------------------
namespace CPUHistogramUtils {
// Edges of an axis given in log10 units: 10^(from + i * (to - from) / nbins), i = 0..nbins.
ST_CXX_API void BinLogX(int nbins, double from, double to, double* edges);
// Counts per bin to a normalised density (divide by bin width, then by the count total).
ST_CXX_API void PMF_to_PDF(int nbins, const double* edges, double* contents);
// Density to y*f(y) (multiply by the bin midpoint).
ST_CXX_API void Prepare_for_Semilog(int nbins, const double* edges, double* contents);
}  // namespace CPUHistogramUtils

// ---------------------------------------------------------------------------------------------
// Tasks and their seeds (ThreadTask.hh:6-31, ThreadAllocation.cc:16-32, ThreadAllocator.cc).
// ---------------------------------------------------------------------------------------------
struct ST_CXX_API ThreadTask {
  std::string fileName;
  int64_t entryPoint = 0;   // first deposit of the track in the file
  int64_t exitPoint = 0;    // one past the last deposit
  int64_t randomSeed = 0;
  int32_t threadID = 0;
  int32_t nOversamples = 1;
  int32_t trackInFile = 0;
};

struct ST_CXX_API ThreadAllocation {
  int32_t threadID = 0;
  int64_t randomSeed = 0;
  int32_t nOversamples = 1;
  std::vector<ThreadTask> tasks;
  // The task seed is the decimal concatenation of the run seed, the thread id and the task's
  // position in the thread (ThreadAllocation.cc:28-31). Returns false if it overflows int64.
  bool AddTask(const ThreadTask& task);
};

struct ST_CXX_API RunConfig {
  std::string type;
  std::string path;
  long firstFile = -1;
  long lastFile = -1;
  long threads = 1;
  long oversamples = 1;
  long randomSeed = -1;
};

// Reads the [Run] keys (ThreadAllocator.cc:29-49). RandomSeed -1 becomes time(NULL).
// Returns an empty string on success or the reason the macro is unusable.
ST_CXX_API std::string ReadRunConfig(const INIReader& reader, RunConfig* cfg);

// Folder enumeration, file limits, one task per track and the contiguous split over threads
// (ThreadAllocator.cc:51-133). Returns an empty string on success or the error text.
ST_CXX_API std::string ReturnThreadAllocations(const RunConfig& cfg, std::vector<ThreadAllocation>* out);

// ---------------------------------------------------------------------------------------------
// Track files. One file holds several tracks as float64 SoA deposits plus the cumulative end
// index of every track (the role of the "Tracks" tree with branches x/y/z [nm], edep [eV] and
// the "Track index" tree, Track.cu:25-31, ThreadAllocator.cc:138-156).
//   offset 0   : char[8]  "STRKv001"
//   offset 8   : uint64   n_deposits
//   offset 16  : uint64   n_tracks
//   offset 24  : uint64   index[n_tracks]   (cumulative end entries)
//   then       : float64  x[n], y[n], z[n], edep[n]
// ---------------------------------------------------------------------------------------------
constexpr const char* kTrackFileExtension = ".strk";
ST_CXX_API bool ReadTrackIndex(const std::string& path, std::vector<uint64_t>* index, uint64_t* n_deposits);
ST_CXX_API bool ReadTrackDeposits(const std::string& path, int64_t begin, int64_t end, double* x, double* y,
                       double* z, double* edep);
ST_CXX_API bool WriteTrackFile(const std::string& path, uint64_t n_tracks, const uint64_t* index,
                    uint64_t n_deposits, const double* x, const double* y, const double* z,
                    const double* edep);

}  // namespace st
