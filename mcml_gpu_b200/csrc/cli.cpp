// cli.cpp -- the MCML_GPU command line, drop-in for the reference's main.cu.
//
//   MCML_GPU sim_set.json input.txt output.txt [-h -R -A -P -AP -B -G # -LS]
//
// Flag semantics, dependency checks, messages and exit codes follow
// main.cu:17-145: usage errors print a message and exit 0, a bad
// configuration exits 1.  Additive flags (ignored by the reference):
//   -S <seed>      fixed XORWOW seed (default time(NULL), transport.cu:72)
//   -T <slots>     RNG subsequences ("photon slots"); default = the
//                  reference's thread count on the selected GPU
//   -grid nr nz dr dz   absorbance grid (default 1000 500 0.01 0.01)
//   -CK <file>     checkpointed first pass: launches of a slice of the slots,
//                  the file brought up to date after each, a run resumes
//                  from it when it exists (<file>.<i> for simulation i > 0)
//   -batch         every simulation of the file in one batched launch
//                  (first pass only: output.txt and summary.json)
#include <cctype>
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/mcml_b200.h"

namespace {

// Values of this CLI's own options (-S, -T, -grid): the whole argument
// must be the number, so a typo is reported instead of read as 0.
bool parse_u64(const char *s, unsigned long long *out) {
  if (!s || !std::isdigit((unsigned char)s[0])) return false;
  errno = 0;
  char *end = nullptr;
  const unsigned long long v = std::strtoull(s, &end, 10);
  if (errno == ERANGE || *end != '\0') return false;
  *out = v;
  return true;
}

bool parse_length(const char *s, float *out) {
  if (!s || !*s) return false;
  errno = 0;
  char *end = nullptr;
  const float v = std::strtof(s, &end);
  if (errno == ERANGE || *end != '\0' || !std::isfinite(v) || !(v > 0.0f)) return false;
  *out = v;
  return true;
}

void show_usage(const std::string &name) {
  const size_t found = name.find_last_of("/\\");
  const std::string exename = name.substr(found + 1);
  std::cerr << "Usage: " << exename << " sim_set.json input.txt output.txt <option(s)>\n"
            << "Options:\n"
            << "\t-h,--help\t Show this help message\n"
            << "\t-R,\t\t Replay the detected photon after first simulation\n"
            << "\t-A,\t\t Output the absorbance array\n"
            << "\t-P,\t\t Output the pathlength for each photon, otherwise output the calculated "
               "average pathlength\n"
            << "\t-AP,\t\t Calaulate and output the average pathlength\n"
            << "\t-B,\t\t Output the pathlength and absorbance file in binary format\n"
            << "\t-LS,\t\t List the GPUs and not run simulation\n"
            << "\t-G,\t\t Select which GPU to run, following by a number start from 0\n"
            << "\t-S,\t\t Seed of the random number generator (default: time(NULL))\n"
            << "\t-T,\t\t Number of photon slots / RNG subsequences (default: reference layout)\n"
            << "\t-grid,\t\t Absorbance grid: nr nz dr dz (default: 1000 500 0.01 0.01)\n"
            << "\t-CK,\t\t Checkpoint file of the first pass, following by a path (resumes if present)\n"
            << "\t-batch,\t\t Run all simulations in one batched launch (no -R)\n"
            << std::endl;
}

int list_gpus(bool print) {
  int n = 0;
  if (mcml_device_count(&n) != MCML_OK || n == 0) {
    std::cout << "ERROR: No CUDA-capable GPU device found\n";
    return 0;
  }
  for (int d = 0; d < n && print; ++d) {
    mcml_device_info info;
    if (mcml_get_device_info(d, &info) != MCML_OK) continue;
    std::cout << "=======================   GPU Infomation  ==========================\n";
    std::printf("Device %d of %d:\t\t%s\n", d + 1, n, info.name);
    std::printf("Compute Capability:\t%d.%d\n", info.major, info.minor);
    std::printf("Global Memory:\t\t%llu B\n", (unsigned long long)info.global_mem);
    std::printf("Number of MPs:\t\t%d\n", info.sm_count);
    std::printf("Max Thread per MP:\t%d\n", info.max_threads_per_sm);
    std::printf("Reference thread layout:\t%llu\n\n",
                (unsigned long long)info.reference_threads);
  }
  return n;
}

void print_banner() {
  std::cout << "******************************" << std::endl;
  std::cout << "*       MCML_GPU K3.02       *" << std::endl;
  std::cout << "*   B200-native mcml_b200    *" << std::endl;
  std::cout << "******************************" << std::endl;
}

}  // namespace

int main(int argc, char *argv[]) {
  bool do_replay = false, do_A = false, do_P = false, do_AP = false, do_B = false;
  int gpu = 0;
  bool have_seed = false;
  unsigned long long seed = 0;
  unsigned long long slots = 0;
  unsigned grid_nr = 0, grid_nz = 0;
  float grid_dr = 0, grid_dz = 0;
  std::string checkpoint;
  bool do_batch = false;

  for (int i = 1; i < argc; i++) {
    const std::string a(argv[i]);
    if (a == "-h") {
      show_usage(argv[0]);
      return 0;
    } else if (a == "-R") {
      do_replay = true;
    } else if (a == "-A") {
      do_A = true;
    } else if (a == "-P") {
      do_P = true;
    } else if (a == "-AP") {
      do_AP = true;
    } else if (a == "-B") {
      do_B = true;
    } else if (a == "-G") {
      if (i + 1 >= argc) {
        std::cout << "GPU selection ERROR!\n";
        return 0;
      }
      int selected = 0;
      try {
        selected = std::stoi(std::string(argv[i + 1]));
      } catch (...) {
        std::cout << "GPU selection ERROR!\n";
        return 0;
      }
      if (selected < 0) {
        std::cout << "GPU selection ERROR!\n";
        return 0;
      }
      gpu = selected;
    } else if (a == "-LS") {
      list_gpus(true);
      return 0;
    } else if (a == "-S") {
      if (i + 1 >= argc || !parse_u64(argv[i + 1], &seed)) {
        std::cout << "-S option needs a seed (an unsigned integer)!\n";
        return 0;
      }
      ++i;
      have_seed = true;
    } else if (a == "-T") {
      if (i + 1 >= argc || !parse_u64(argv[i + 1], &slots)) {
        std::cout << "-T option needs a slot count (an unsigned integer, 0 for automatic)!\n";
        return 0;
      }
      ++i;
    } else if (a == "-grid") {
      unsigned long long nr = 0, nz = 0;
      if (i + 4 >= argc || !parse_u64(argv[i + 1], &nr) || !parse_u64(argv[i + 2], &nz) ||
          nr == 0 || nz == 0 || nr > 0x7fffffffull || nz > 0x7fffffffull ||
          !parse_length(argv[i + 3], &grid_dr) || !parse_length(argv[i + 4], &grid_dz)) {
        std::cout << "-grid option needs nr nz dr dz (two positive cell counts, two positive "
                     "cell sizes in cm)!\n";
        return 0;
      }
      grid_nr = (unsigned)nr;
      grid_nz = (unsigned)nz;
      i += 4;
    } else if (a == "-CK") {
      if (i + 1 >= argc) {
        std::cout << "-CK option needs a checkpoint file name!\n";
        return 0;
      }
      checkpoint = argv[++i];
    } else if (a == "-batch") {
      do_batch = true;
    }
  }

  if (argc < 4) {
    show_usage(argv[0]);
    return 0;
  }
  if (do_replay && !do_P) do_AP = true;
  if (do_P && !do_replay) {
    std::cout << "-P option only work with -R option!\n";
    return 0;
  }
  if (do_A && !do_replay) {
    std::cout << "-A option only work with -R option!\n";
    return 0;
  }
  if (do_AP && !do_replay) {
    std::cout << "-AP option only work with -R option!\n";
    return 0;
  }
  if (do_B && !(do_P || do_A)) {
    std::cout << "-B option only work with -P or -A option!\n";
    return 0;
  }
  if (do_batch && (do_replay || !checkpoint.empty())) {
    std::cout << "-batch option does not work with -R or -CK option!\n";
    return 0;
  }

  int n_sims = 0;
  if (mcml_parse_config(argv[1], argv[2], nullptr, 0, &n_sims) != MCML_OK || n_sims <= 0) {
    std::cout << mcml_last_error() << "\n";
    std::printf("Something wrong with read_simulation_data!\n");
    return 1;
  }
  std::vector<mcml_sim> sims(n_sims);
  if (mcml_parse_config(argv[1], argv[2], sims.data(), n_sims, &n_sims) != MCML_OK) {
    std::cout << mcml_last_error() << "\n";
    std::printf("Something wrong with read_simulation_data!\n");
    return 1;
  }

  print_banner();
  const int gpu_count = list_gpus(true);
  if (gpu >= gpu_count) {
    std::cout << "GPU selection ERROR!\n";
    return 0;
  }
  std::cout << "GPU " << gpu << " is selected\n";

  if (!have_seed) seed = (unsigned long long)time(NULL);
  uint32_t flags = 0;
  if (do_replay) flags |= MCML_OUT_REPLAY;
  if (do_A) flags |= MCML_OUT_ABSORBANCE;
  if (do_P) flags |= MCML_OUT_PATHLENGTH;
  if (do_AP) flags |= MCML_OUT_AVERAGE_PL;
  if (do_B) flags |= MCML_OUT_BINARY;

  const auto t_all = std::chrono::steady_clock::now();
  if (do_batch) {
    mcml_batch_opts bo{};
    bo.seed = seed;
    bo.device = gpu;
    mcml_batch *b = nullptr;
    int rc = mcml_batch_create(sims.data(), n_sims, &bo, &b);
    if (rc == MCML_OK) rc = mcml_batch_autotune(b, 1.0 / 64, nullptr);
    std::vector<mcml_result> res(n_sims);
    const auto t0 = std::chrono::steady_clock::now();
    if (rc == MCML_OK) rc = mcml_batch_run(b, res.data());
    const auto t1 = std::chrono::steady_clock::now();
    if (rc != MCML_OK) {
      std::printf("Error: %s (%s)\n", mcml_strerror(rc), mcml_last_error());
      if (b) mcml_batch_destroy(b);
      return 1;
    }
    mcml_batch_destroy(b);
    mcml_device_info info{};
    mcml_get_device_info(gpu, &info);
    const double sim_s = std::chrono::duration<double>(t1 - t0).count();
    for (int i = 0; i < n_sims; i++) {
      std::vector<uint64_t> det(res[i].num_sds);
      for (unsigned d = 0; d < res[i].num_sds; d++) det[d] = res[i].detected[d];
      mcml_host_data hd{};
      hd.photons = sims[i].number_photons;
      hd.detected = det.data();
      hd.weight_sum = res[i].weight_sum;
      hd.gpu_name = info.name;
      rc = mcml_write_host_outputs(&sims[i], &hd, "", argv[3], 0, sim_s / n_sims, 0.0);
      if (rc != MCML_OK) {
        std::printf("Error: %s (%s)\n", mcml_strerror(rc), mcml_last_error());
        return 1;
      }
      std::printf("simulation %d:", i);
      for (unsigned d = 0; d < res[i].num_sds; d++)
        std::printf(" SDS %u %.6e +- %.2e;", d + 1, res[i].reflectance[d], res[i].std_error[d]);
      std::printf("\n");
    }
    std::printf("Simulation time: %.2f sec\n",
                std::chrono::duration<double>(std::chrono::steady_clock::now() - t_all).count());
    return 0;
  }
  for (int i = 0; i < n_sims; i++) {
    std::printf("simulating %d\n", i);
    mcml_opts opts{};
    opts.seed = seed;
    opts.slots = slots;
    opts.device = gpu;
    opts.grid_nr = grid_nr;
    opts.grid_nz = grid_nz;
    opts.grid_dr = grid_dr;
    opts.grid_dz = grid_dz;
    mcml_ctx *ctx = nullptr;
    int rc = mcml_create(&sims[i], &opts, &ctx);
    if (rc != MCML_OK) {
      std::printf("Error: %s (%s)\n", mcml_strerror(rc), mcml_last_error());
      return 1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    mcml_result res{};
    if (checkpoint.empty()) {
      rc = mcml_run(ctx, &res);
    } else {
      const std::string path = i == 0 ? checkpoint : checkpoint + "." + std::to_string(i);
      mcml_checkpoint_opts ck{};
      ck.path = path.c_str();
      rc = mcml_run_checkpointed(ctx, &ck, &res);
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (rc != MCML_OK) {
      std::printf("Error: %s (%s)\n", mcml_strerror(rc), mcml_last_error());
      mcml_destroy(ctx);
      return 1;
    }
    const double sim_s = std::chrono::duration<double>(t1 - t0).count();
    std::printf("Number of photons terminated %llu, photon deteced number for SDSs:",
                (unsigned long long)res.photons);
    for (unsigned d = 0; d < res.num_sds; d++) std::printf("\t%llu,", (unsigned long long)res.detected[d]);
    std::printf("\nfinish first run, cost %.2f secs\n", sim_s);
    double replay_s = 0.0;
    if (do_replay) {
      const auto r0 = std::chrono::steady_clock::now();
      rc = mcml_replay(ctx, nullptr);
      const auto r1 = std::chrono::steady_clock::now();
      if (rc != MCML_OK) {
        std::printf("Error: %s (%s)\n", mcml_strerror(rc), mcml_last_error());
        mcml_destroy(ctx);
        return 1;
      }
      replay_s = std::chrono::duration<double>(r1 - r0).count();
    }
    rc = mcml_write_outputs(ctx, "", argv[3], flags, sim_s, replay_s);
    if (rc != MCML_OK) {
      std::printf("Error: %s (%s)\n", mcml_strerror(rc), mcml_last_error());
      mcml_destroy(ctx);
      return 1;
    }
    if (do_replay) std::printf("finish replay, cost %.2f secs\n", replay_s);
    for (unsigned d = 0; d < res.num_sds; d++)
      std::printf("SDS %u: reflectance %.6e +- %.2e (1 SE)\n", d + 1, res.reflectance[d],
                  res.std_error[d]);
    mcml_destroy(ctx);
  }
  const auto t_end = std::chrono::steady_clock::now();
  std::printf("Simulation time: %.2f sec\n",
              std::chrono::duration<double>(t_end - t_all).count());
  return 0;
}
