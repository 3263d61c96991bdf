// `supertrack [macro.ini]` — the command-line run of SuperTrack.cu:9-36: reads the macro
// (default ../macros/default.ini), runs every task of the track folder on GPU 0 and writes
// <[Output] Path><NamePrefix><seed>.csv and .json.
#include <chrono>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/supertrack_b200.h"

int main(int argc, char** argv) {
  const auto t0 = std::chrono::steady_clock::now();
  std::string ini = "../macros/default.ini";
  if (argc == 2) ini = argv[1];
  char err[1024] = {0};
  st_run_info info;
  const st_status s = st_run_macro(ini.c_str(), 0, 1, nullptr, nullptr, 0, &info, err, sizeof(err));
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (s != ST_OK) {
    std::fprintf(stderr, "SuperTrack failed (%s): %s\n", st_status_string(s), err);
    return 1;
  }
  std::printf("SuperTrack: %lld tracks x %lld oversamples (%lld deposits), seed %lld\n",
              (long long)info.n_tracks, (long long)info.n_oversamples, (long long)info.deposits,
              (long long)info.random_seed);
  std::printf("SuperTrack concluding after: %.3f seconds.\n", secs);
  return 0;
}
