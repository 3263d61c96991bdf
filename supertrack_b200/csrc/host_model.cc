#include "host_model.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <filesystem>
#include <fstream>
#include <sstream>

namespace st {

// ---------------------------------------------------------------------------------------------
// INIReader
// ---------------------------------------------------------------------------------------------
namespace {

std::string rstrip(const std::string& s) {
  size_t e = s.size();
  while (e > 0 && std::isspace((unsigned char)s[e - 1])) --e;
  return s.substr(0, e);
}

size_t lskip(const std::string& s, size_t pos) {
  while (pos < s.size() && std::isspace((unsigned char)s[pos])) ++pos;
  return pos;
}

// Position of the first character of `chars` or of an inline ';' comment that follows
// whitespace, scanning from pos; npos-like s.size() when neither occurs.
size_t find_chars_or_comment(const std::string& s, size_t pos, const char* chars) {
  bool was_space = false;
  for (size_t i = pos; i < s.size(); ++i) {
    const char c = s[i];
    if (chars && std::strchr(chars, c) && c != '\0') return i;
    if (was_space && c == ';') return i;
    was_space = std::isspace((unsigned char)c) != 0;
  }
  return s.size();
}

}  // namespace

INIReader::INIReader(const std::string& filename) {
  std::ifstream f(filename, std::ios::binary);
  if (!f) { _error = -1; return; }
  std::stringstream ss;
  ss << f.rdbuf();
  ParseText(ss.str());
}

INIReader INIReader::FromString(const std::string& text) {
  INIReader r;
  r.ParseText(text);
  return r;
}

std::string INIReader::MakeKey(const std::string& section, const std::string& name) {
  std::string key = section + "=" + name;
  std::transform(key.begin(), key.end(), key.begin(), [](unsigned char c) { return std::tolower(c); });
  return key;
}

void INIReader::ParseText(const std::string& text) {
  std::string section;
  std::string prev_name;
  int lineno = 0;
  size_t pos = 0;
  auto add = [&](const std::string& sec, const std::string& name, const std::string& value) {
    const std::string key = MakeKey(sec, name);
    std::string& slot = _values[key];
    if (!slot.empty()) slot += "\n";
    slot += value;
    _sections.insert(sec);
  };
  while (pos < text.size()) {
    size_t nl = text.find('\n', pos);
    std::string line = text.substr(pos, nl == std::string::npos ? std::string::npos : nl - pos + 1);
    pos = (nl == std::string::npos) ? text.size() : nl + 1;
    ++lineno;
    if (lineno == 1 && line.size() >= 3 && (unsigned char)line[0] == 0xEF &&
        (unsigned char)line[1] == 0xBB && (unsigned char)line[2] == 0xBF) {
      line = line.substr(3);
    }
    const std::string stripped = rstrip(line);
    const size_t start = lskip(stripped, 0);
    if (start >= stripped.size()) continue;  // blank line
    const char c0 = stripped[start];
    if (c0 == ';' || c0 == '#') continue;
    if (!prev_name.empty() && start > 0) {
      // indented non-blank line: continuation of the previous value
      size_t end = find_chars_or_comment(stripped, start, nullptr);
      add(section, prev_name, rstrip(stripped.substr(start, end - start)));
      continue;
    }
    if (c0 == '[') {
      const size_t end = find_chars_or_comment(stripped, start + 1, "]");
      if (end < stripped.size() && stripped[end] == ']') {
        section = stripped.substr(start + 1, end - start - 1);
        prev_name.clear();
      } else if (!_error) {
        _error = lineno;
      }
      continue;
    }
    const size_t end = find_chars_or_comment(stripped, start, "=:");
    if (end < stripped.size() && (stripped[end] == '=' || stripped[end] == ':')) {
      const std::string name = rstrip(stripped.substr(start, end - start));
      const size_t vstart = lskip(stripped, end + 1);
      const size_t vend = find_chars_or_comment(stripped, vstart, nullptr);
      const std::string value = rstrip(stripped.substr(vstart, vend - vstart));
      prev_name = name;
      add(section, name, value);
    } else if (!_error) {
      _error = lineno;
    }
  }
}

std::string INIReader::Get(const std::string& section, const std::string& name,
                           const std::string& default_value) const {
  const auto it = _values.find(MakeKey(section, name));
  return it == _values.end() ? default_value : it->second;
}

bool INIReader::Has(const std::string& section, const std::string& name) const {
  return _values.count(MakeKey(section, name)) != 0;
}

long INIReader::GetInteger(const std::string& section, const std::string& name,
                           long default_value) const {
  const std::string v = Get(section, name, "");
  const char* s = v.c_str();
  char* end;
  const long n = std::strtol(s, &end, 0);
  return end > s ? n : default_value;
}

double INIReader::GetReal(const std::string& section, const std::string& name,
                          double default_value) const {
  const std::string v = Get(section, name, "");
  const char* s = v.c_str();
  char* end;
  const double n = std::strtod(s, &end);
  return end > s ? n : default_value;
}

float INIReader::GetFloat(const std::string& section, const std::string& name,
                          float default_value) const {
  const std::string v = Get(section, name, "");
  const char* s = v.c_str();
  char* end;
  const float n = std::strtof(s, &end);
  return end > s ? n : default_value;
}

bool INIReader::GetBoolean(const std::string& section, const std::string& name,
                           bool default_value) const {
  std::string v = Get(section, name, "");
  std::transform(v.begin(), v.end(), v.begin(), [](unsigned char c) { return std::tolower(c); });
  if (v == "true" || v == "yes" || v == "on" || v == "1") return true;
  if (v == "false" || v == "no" || v == "off" || v == "0") return false;
  return default_value;
}

// ---------------------------------------------------------------------------------------------
// Bin edges
// ---------------------------------------------------------------------------------------------
void LinSpace(float bottom, float top, int nbins, double* bins) {
  const double width = (top - bottom) / (nbins);  // float subtraction and division
  for (int i = 0; i <= nbins; i++) bins[i] = bottom + (i * width);
}

void LogSpace(float bottom, float top, int nbins, double* bins) {
  const float bottom_order_mag = (float)std::log10((double)bottom);
  const float top_order_mag = (float)std::log10((double)top);
  const double width = (top_order_mag - bottom_order_mag) / (nbins);
  for (int i = 0; i <= nbins; i++) bins[i] = std::pow(10.0, bottom_order_mag + (i * width));
}

bool MakeEdges(int type, int nbins, float lower, float upper, std::vector<double>* edges) {
  if (nbins < 1 || nbins > (1 << 26)) return false;
  edges->assign((size_t)nbins + 1, 0.0);
  if (type == 0) LinSpace(lower, upper, nbins, edges->data());
  else if (type == 1) LogSpace(lower, upper, nbins, edges->data());
  else return false;
  for (int i = 0; i <= nbins; ++i) {
    if (!std::isfinite((*edges)[i])) return false;
    if (i > 0 && !((*edges)[i] > (*edges)[i - 1])) return false;
  }
  return true;
}

// ---------------------------------------------------------------------------------------------
// Tasks
// ---------------------------------------------------------------------------------------------
bool ThreadAllocation::AddTask(const ThreadTask& task) {
  const size_t ntasks = tasks.size();
  tasks.push_back(task);
  ThreadTask& t = tasks.back();
  t.threadID = threadID;
  t.nOversamples = nOversamples;
  std::stringstream cs;
  cs << randomSeed << threadID << ntasks;
  const std::string s = cs.str();
  errno = 0;
  char* end = nullptr;
  const long long v = std::strtoll(s.c_str(), &end, 10);
  if (errno == ERANGE || end == s.c_str()) return false;
  t.randomSeed = v;
  return true;
}

std::string ReadRunConfig(const INIReader& reader, RunConfig* cfg) {
  cfg->type = reader.Get("Run", "Type", "");
  if (cfg->type != "Folder")
    return "Macro file error: ([Run], Type) does not = folder. Only analysis runs over folders are supported.";
  cfg->path = reader.Get("Run", "Path", "");
  if (cfg->path.empty()) return "Macro file error: ([Run], Folder) not defined.";
  cfg->firstFile = reader.GetInteger("Run", "FirstFile", -1);
  cfg->lastFile = reader.GetInteger("Run", "LastFile", -1);
  cfg->threads = reader.GetInteger("Run", "Threads", 1);
  cfg->oversamples = reader.GetInteger("Run", "Oversamples", 1);
  cfg->randomSeed = reader.GetInteger("Run", "RandomSeed", -1);
  if (cfg->randomSeed == -1) cfg->randomSeed = (long)time(nullptr);
  if (cfg->threads < 1) return "Macro file error: ([Run], Threads) must be at least 1.";
  if (cfg->oversamples < 0 || cfg->oversamples > INT_MAX)
    return "Macro file error: ([Run], Oversamples) out of range.";
  return "";
}

std::string ReturnThreadAllocations(const RunConfig& cfg, std::vector<ThreadAllocation>* out) {
  namespace fs = std::filesystem;
  std::vector<std::string> files;
  std::error_code ec;
  fs::directory_iterator it(cfg.path, ec);
  if (ec) return "Cannot open track folder: " + cfg.path;
  for (const auto& e : it)
    if (e.path().extension() == kTrackFileExtension) files.push_back(e.path().string());
  std::sort(files.begin(), files.end());

  long lo = cfg.firstFile, hi = cfg.lastFile;
  const long folderSize = (long)files.size();
  if (lo == -1 && hi == -1) {
    lo = 1;
    hi = folderSize;
  } else if (hi < lo) {
    return "Lower file limit greater than upper file limit. Aborting.";
  } else if (hi > folderSize) {
    return "Upper file limit greater than number of files. Aborting.";
  } else if (lo < 1) {
    return "Lower file limit less than 1. Aborting.";
  }

  std::vector<ThreadTask> tasks;
  for (long i = lo; i <= hi; ++i) {
    std::vector<uint64_t> index;
    uint64_t nd = 0;
    if (!ReadTrackIndex(files[i - 1], &index, &nd)) return "Cannot read track file: " + files[i - 1];
    uint64_t start = 0;
    for (size_t k = 0; k < index.size(); ++k) {
      ThreadTask t;
      t.fileName = files[i - 1];
      t.entryPoint = (int64_t)start;
      t.exitPoint = (int64_t)index[k];
      t.trackInFile = (int32_t)k;
      tasks.push_back(t);
      start = index[k];
    }
  }

  long numThreads = cfg.threads;
  if ((long)tasks.size() < numThreads) numThreads = (long)tasks.size();
  out->clear();
  if (numThreads == 0) return "";
  const long perThread = (long)tasks.size() / numThreads;
  const long remainder = (long)tasks.size() % numThreads;
  size_t current = 0;
  for (long i = 0; i < numThreads; ++i) {
    ThreadAllocation a;
    a.threadID = (int32_t)i;
    a.randomSeed = cfg.randomSeed;
    a.nOversamples = (int32_t)cfg.oversamples;
    out->push_back(a);
    const long n = perThread + (i < remainder ? 1 : 0);
    for (long j = 0; j < n; ++j) {
      if (!out->back().AddTask(tasks[current])) return "Task seed overflows a 64-bit integer.";
      ++current;
    }
  }
  return "";
}

// ---------------------------------------------------------------------------------------------
// Track files
// ---------------------------------------------------------------------------------------------
namespace {
const char kMagic[8] = {'S', 'T', 'R', 'K', 'v', '0', '0', '1'};
}

bool ReadTrackIndex(const std::string& path, std::vector<uint64_t>* index, uint64_t* n_deposits) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  char magic[8];
  uint64_t hdr[2];
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kMagic, 8) == 0 &&
            std::fread(hdr, 8, 2, f) == 2;
  if (ok) {
    *n_deposits = hdr[0];
    index->resize(hdr[1]);
    ok = hdr[1] == 0 || std::fread(index->data(), 8, hdr[1], f) == hdr[1];
    uint64_t prev = 0;
    for (size_t i = 0; ok && i < index->size(); ++i) {
      if ((*index)[i] < prev || (*index)[i] > hdr[0]) ok = false;
      prev = (*index)[i];
    }
  }
  std::fclose(f);
  return ok;
}

bool ReadTrackDeposits(const std::string& path, int64_t begin, int64_t end, double* x, double* y,
                       double* z, double* edep) {
  std::vector<uint64_t> index;
  uint64_t n = 0;
  if (!ReadTrackIndex(path, &index, &n)) return false;
  if (begin < 0 || end < begin || (uint64_t)end > n) return false;
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  const int64_t base = 24 + 8 * (int64_t)index.size();
  const int64_t cnt = end - begin;
  double* dst[4] = {x, y, z, edep};
  bool ok = true;
  for (int a = 0; a < 4 && ok; ++a) {
    const int64_t off = base + 8 * ((int64_t)n * a + begin);
    ok = std::fseek(f, off, SEEK_SET) == 0 &&
         (cnt == 0 || std::fread(dst[a], 8, (size_t)cnt, f) == (size_t)cnt);
  }
  std::fclose(f);
  return ok;
}

bool WriteTrackFile(const std::string& path, uint64_t n_tracks, const uint64_t* index,
                    uint64_t n_deposits, const double* x, const double* y, const double* z,
                    const double* edep) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const uint64_t hdr[2] = {n_deposits, n_tracks};
  bool ok = std::fwrite(kMagic, 1, 8, f) == 8 && std::fwrite(hdr, 8, 2, f) == 2 &&
            (n_tracks == 0 || std::fwrite(index, 8, n_tracks, f) == n_tracks);
  const double* src[4] = {x, y, z, edep};
  for (int a = 0; a < 4 && ok; ++a)
    ok = n_deposits == 0 || std::fwrite(src[a], 8, n_deposits, f) == n_deposits;
  ok = (std::fclose(f) == 0) && ok;
  return ok;
}

// ---------------------------------------------------------------------------------------------
// Spectrum post-processing (utils.cc:37-117)
// ---------------------------------------------------------------------------------------------
namespace CPUHistogramUtils {
namespace {
// TAxis::GetBinLowEdge of an axis built from explicit edges: the edge for bins 1..nbins+1,
// the equidistant extrapolation below (or above) that range.
double low_edge(int nbins, const double* edges, int bin) {
  if (bin < 1 || bin > nbins + 1) {
    const double w = (edges[nbins] - edges[0]) / (double)nbins;
    return edges[0] + (double)(bin - 1) * w;
  }
  return edges[bin - 1];
}
}  // namespace

void BinLogX(int nbins, double from, double to, double* edges) {
  const double width = (to - from) / nbins;
  for (int i = 0; i <= nbins; i++) edges[i] = std::pow(10.0, from + i * width);
}

void PMF_to_PDF(int nbins, const double* edges, double* contents) {
  float normalization = 0;
  for (int i = 0; i < nbins; i++) {
    const double value = contents[i];
    const double low = low_edge(nbins, edges, i);
    const double high = low_edge(nbins, edges, i + 1);
    contents[i] = value / (high - low);
    normalization += value;
  }
  for (int i = 0; i < nbins; i++) contents[i] = contents[i] / normalization;
}

void Prepare_for_Semilog(int nbins, const double* edges, double* contents) {
  for (int i = 0; i < nbins; i++) {
    const double low = low_edge(nbins, edges, i);
    const double high = low_edge(nbins, edges, i + 1);
    contents[i] = contents[i] * ((high + low) / 2);
  }
}
}  // namespace CPUHistogramUtils

}  // namespace st
