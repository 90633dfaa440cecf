// hello -- drop-in command line of the k-NN graph builder.
//
//   hello <input_file> <output_file> <k> <trees> <leaf_size> <propagations>
//         <EUCLIDEAN|TAXICAB|COSINE> <gpu_id[,gpu_id...]> <cluster: T/F> [--debug]
//
// Same argument order, messages and exit codes as the reference's main.cpp
// (main.cpp:8-124): 1 wrong argument count, 2 unknown metric, 3 device not
// present, 4 compute capability 1.x, 5 no CUDA GPU, 7 input not readable,
// 8 initialisation failed, 9 deinitialisation failed.  Input is the reference's
// CSV (README.md:31-47, loadData euclideandistancematrixgpu.cu:2712-2757), parsed
// here by several threads; output is its binary layout (saveResultToResultFile,
// .cu:2908-2978) with the VALIDATION and DEBUG side files.  The points are
// normalised as the reference's calculate() does (.cu:2869-2875) before the
// graph is built by knn_build on the first listed device.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <thread>
#include <vector>

#include "knn.h"

namespace {

void usage() {
  std::cout << "Wrong number of arguments!\n";
  std::cout << "Proper launching: hello.exe <input_file> <output_file> <number_of_neighbours> "
               "<number_of_trees> <number_of_elements_in_leaf> <number_of_propagations> "
               "<distance_Algorithm> <id_gpu> <cluster: T/F> <--debug>\n";
  std::cout << "Example launching: hello.exe input.csv output.csv 2 10 10 10 EUCLIDEAN 1 T\n";
  std::cout << "Example launching: hello.exe input.csv output.csv 2 10 10 10 EUCLIDEAN 1 T --debug\n";
  std::cout << "Available distance algorithms: EUCLIDEAN TAXICAB COSINE\n";
  std::cout << "Attention!\n";
  std::cout << "Delimeter -> ,\n";
  std::cout << "If file has cluster (at the end of line) you should run program with cluster set "
               "T, otherwise F\n";
}

// One CSV point line [s, e): tokens split on ',' (empty tokens skipped, as
// strtok does), each parsed like atof (leading blanks, longest numeric
// prefix, 0 when none) and narrowed to float; with `klaster` the last token is
// the cluster id and is not a feature.  Tokens are copied into a terminated
// buffer first so that the parse cannot run past the token.
void parse_line(const char* s, const char* e, int d, bool klaster, float* row) {
  int ntok = 0;
  for (const char* p = s; p < e;) {  // tokens on the line
    while (p < e && *p == ',') ++p;
    if (p >= e) break;
    ++ntok;
    while (p < e && *p != ',') ++p;
  }
  const int nfeat = std::min(klaster && ntok > 0 ? ntok - 1 : ntok, d);
  char buf[128];
  const char* p = s;
  for (int i = 0; i < nfeat; ++i) {
    while (*p == ',') ++p;
    const char* q = p;
    while (q < e && *q != ',') ++q;
    const size_t len = std::min<size_t>(q - p, sizeof(buf) - 1);
    std::memcpy(buf, p, len);
    buf[len] = 0;
    row[i] = (float)std::atof(buf);
    p = q;
  }
}

// The whole file in one buffer; the point lines after the two header lines
// are cut into one newline-aligned byte range per thread, each thread counts
// its lines, and after a prefix sum parses them into their rows (at most n;
// missing lines and values stay 0, as in the reference's zero-filled table).
bool load_csv(const std::string& path, int64_t n, int d, bool klaster, std::vector<float>& x) {
  std::FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  std::vector<char> text;
  if (std::fseek(f, 0, SEEK_END) == 0) {
    const long size = std::ftell(f);
    if (size > 0) text.resize((size_t)size);
    std::fseek(f, 0, SEEK_SET);
  }
  const size_t got = text.empty() ? 0 : std::fread(text.data(), 1, text.size(), f);
  std::fclose(f);
  text.resize(got);
  const char* const b = text.data();
  const char* const e = b + text.size();
  const char* body = b;
  for (int h = 0; h < 2 && body < e; ++h) {
    const char* nl = static_cast<const char*>(std::memchr(body, '\n', e - body));
    body = nl ? nl + 1 : e;
  }
  x.assign((size_t)n * d, 0.0f);
  const unsigned hw = std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  const size_t span = (size_t)(e - body);
  std::vector<const char*> cut(hw + 1, e);
  cut[0] = body;
  for (unsigned t = 1; t < hw; ++t) {  // range t starts after the newline at or past its share
    const char* p = body + span * t / hw;
    if (p < cut[t - 1]) p = cut[t - 1];
    const char* nl = p > body ? static_cast<const char*>(std::memchr(p - 1, '\n', e - (p - 1))) : nullptr;
    cut[t] = p == body ? body : (nl ? nl + 1 : e);
  }
  auto lines_in = [](const char* p, const char* q) {
    int64_t c = 0;
    while (p < q) {
      const char* nl = static_cast<const char*>(std::memchr(p, '\n', q - p));
      ++c;
      p = nl ? nl + 1 : q;
    }
    return c;
  };
  std::vector<int64_t> first(hw + 1, 0);
  {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < hw; ++t)
      pool.emplace_back([&, t] { first[t + 1] = lines_in(cut[t], cut[t + 1]); });
    for (auto& th : pool) th.join();
  }
  for (unsigned t = 0; t < hw; ++t) first[t + 1] += first[t];
  std::vector<std::thread> pool;
  for (unsigned t = 0; t < hw; ++t) {
    if (first[t] >= n) break;
    pool.emplace_back([&, t] {
      int64_t row = first[t];
      for (const char* p = cut[t]; p < cut[t + 1] && row < n; ++row) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', cut[t + 1] - p));
        const char* q = nl ? nl : cut[t + 1];
        parse_line(p, q, d, klaster, x.data() + (size_t)row * d);
        p = nl ? nl + 1 : cut[t + 1];
      }
    });
  }
  for (auto& th : pool) th.join();
  return true;
}

bool save_result(const std::string& out, const std::vector<int32_t>& idx, const std::vector<float>& dist,
                 int64_t n, int k, int metric, bool debug) {
  std::ofstream ofs(out, std::ofstream::trunc | std::ofstream::binary);
  std::ofstream dbg;
  if (debug) dbg.open(out + "DEBUG", std::ofstream::trunc | std::ofstream::binary);
  std::ofstream val(out + "VALIDATION", std::ofstream::trunc | std::ofstream::binary);
  if (!ofs.is_open()) {
    std::cout << "Can not open the file for saving result.\n";
    return false;
  }
  ofs << n << ";" << k << ";" << sizeof(int64_t) << "\n";
  const int64_t magic = 0x01020304;
  ofs.write(reinterpret_cast<const char*>(&magic), sizeof(magic));
  std::vector<char> rec((size_t)k * 8);
  for (int64_t i = 0; i < n; ++i) {
    for (int s = 0; s < k; ++s) {
      const float dv = dist[(size_t)i * k + s];
      // stored distance: L2, sqrt(L1) (.cu:567-570), or cosine similarity (.cu:1007)
      float stored = dv;
      if (metric == KNN_METRIC_TAXICAB) stored = std::sqrt(dv);
      else if (metric == KNN_METRIC_COSINE) stored = (float)(1.0 - (double)dv);
      const int32_t id = idx[(size_t)i * k + s];
      std::memcpy(rec.data() + (size_t)s * 8, &id, 4);
      std::memcpy(rec.data() + (size_t)s * 8 + 4, &stored, 4);
      if (dbg.is_open()) dbg << "NEAR: <" << i << ", " << id << ">(" << stored << ") ";
    }
    ofs.write(rec.data(), (std::streamsize)rec.size());
    if (dbg.is_open()) dbg << ";\n";
  }
  if (val.is_open()) val << "Everything is OK.";
  return true;
}

// Knobs the reference does not have come from the environment so that the
// positional command line stays the reference's:
//   ACKNN_PRECISION  fp32 (default) | bf16 | f16   leaf blocks in FP32, or in BF16 / FP16
//                    tensor-core tiles + FP32 re-rank
//   ACKNN_SPLITS     median (default) | reference | learned
//   ACKNN_SEED       unsigned integer, default 0
//   ACKNN_TIMING     1: report the wall time of CSV ingest, build and file
//                    write on stderr (stdout stays the reference's)
// An unknown value is reported and fails the initialisation (exit code 8).
bool env_knobs(knn_options& opt, uint64_t& seed) {
  if (const char* v = std::getenv("ACKNN_PRECISION")) {
    const std::string s = v;
    if (s == "fp32") opt.precision = KNN_PREC_FP32;
    else if (s == "bf16") opt.precision = KNN_PREC_BF16_RERANK;
    else if (s == "f16") opt.precision = KNN_PREC_F16_RERANK;
    else {
      std::cout << "ACKNN_PRECISION must be fp32, bf16 or f16\n";
      return false;
    }
  }
  if (const char* v = std::getenv("ACKNN_SPLITS")) {
    const std::string s = v;
    if (s == "median") opt.split_rule = KNN_SPLIT_MEDIAN;
    else if (s == "reference") opt.split_rule = KNN_SPLIT_REFERENCE;
    else if (s == "learned") opt.learned_splits = 1;
    else {
      std::cout << "ACKNN_SPLITS must be median, reference or learned\n";
      return false;
    }
  }
  if (const char* v = std::getenv("ACKNN_SEED")) {
    char* end = nullptr;
    seed = std::strtoull(v, &end, 10);
    if (*v == '\0' || *v == '-' || *end != '\0') {
      std::cout << "ACKNN_SEED must be an unsigned integer\n";
      return false;
    }
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 10 && argc != 11) {
    usage();
    return 1;
  }
  const std::string input = argv[1], output = argv[2];
  const int k = std::atoi(argv[3]);
  const int trees = std::atoi(argv[4]);
  const int leaf = std::atoi(argv[5]);
  const int props = std::atoi(argv[6]);
  const std::string mname = argv[7];
  int metric;
  if (mname == "EUCLIDEAN") metric = KNN_METRIC_EUCLIDEAN;
  else if (mname == "TAXICAB") metric = KNN_METRIC_TAXICAB;
  else if (mname == "COSINE") metric = KNN_METRIC_COSINE;
  else {
    std::cout << "Wrong distance algorithm!\n";
    std::cout << "Available distance algorithms: EUCLIDEAN TAXICAB COSINE\n";
    return 2;
  }
  std::vector<int> devices;
  {
    std::string list = argv[8];
    size_t p = 0;
    while (p <= list.size()) {
      size_t q = list.find(',', p);
      if (q == std::string::npos) q = list.size();
      if (q > p) devices.push_back(std::atoi(list.substr(p, q - p).c_str()));
      p = q + 1;
    }
  }
  for (int dev : devices) {
    int32_t major = 0, minor = 0;
    const int rc = knn_device_capability(dev, &major, &minor);
    if (rc != KNN_OK) {
      std::cout << "Device with id " << dev << " is not located in this computer\n";
      return 3;
    }
    if (major == 1) {
      std::cout << "Device with id " << dev
                << " can not be use because Compute Capability. Required at least 2.0 Compute "
                   "Capability, your GPU has "
                << major << "." << minor << "\n";
      return 4;
    }
    if (major == 9999) {
      std::cout << "This computer does not have any GPU with CUDA\n";
      return 5;
    }
  }
  const bool klaster = std::string(argv[9]) == "T";
  const bool debug = argc == 11 && std::string(argv[10]) == "--debug";

  std::ifstream head(input);
  if (!head.is_open()) {
    std::cout << "Error opening the file\n";
    return 7;
  }
  std::string line;
  std::getline(head, line);
  const int64_t n = std::atoi(line.c_str());
  std::getline(head, line);
  const int d = std::atoi(line.c_str());
  head.close();

  const char* timing_env = std::getenv("ACKNN_TIMING");
  const bool timing = timing_env && std::string(timing_env) == "1";
  using clock = std::chrono::steady_clock;
  const auto t_load = clock::now();
  std::vector<float> x;
  if (devices.empty() || n < 1 || d < 1 || !load_csv(input, n, d, klaster, x)) {
    std::cout << "Initialization failed.\n";
    return 8;
  }
  const double load_ms = std::chrono::duration<double, std::milli>(clock::now() - t_load).count();
  std::cout << "The datafile has been opened\n";
  std::cout << "I begin analysis.\n";
  knn_options opt;
  knn_default_options(&opt);
  opt.device = devices[0];
  uint64_t seed = 0;
  if (!env_knobs(opt, seed)) {
    std::cout << "Initialization failed.\n";
    return 8;
  }
  std::vector<int32_t> idx((size_t)n * (k > 0 ? k : 1));
  std::vector<float> dist((size_t)n * (k > 0 ? k : 1));
  const auto t0 = std::chrono::steady_clock::now();
  int rc = knn_normalize_reference(x.data(), n, d);
  if (rc == KNN_OK)
    rc = knn_build_ex(nullptr, x.data(), n, d, k, trees, leaf, props, metric, seed, idx.data(),
                      dist.data(), &opt, nullptr);
  const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (rc != KNN_OK) {
    std::cout << "k-NN graph build failed: " << knn_status_string(rc) << " (" << knn_last_error() << ")\n";
    return 8;
  }
  std::cout << "The device " << devices[0] << ": has done task in: " << ms << " ms\n";
  std::cout << "I am writing the solution to a file.\n";
  const auto t_write = clock::now();
  if (!save_result(output, idx, dist, n, k, metric, debug)) {
    std::cout << "Deinitialization failed.\n";
    return 9;
  }
  if (timing) {
    const double write_ms = std::chrono::duration<double, std::milli>(clock::now() - t_write).count();
    std::fprintf(stderr, "acknn timing: load_ms=%.1f build_ms=%.1f write_ms=%.1f threads=%u\n", load_ms, ms,
                 write_ms, std::max(1u, std::min(64u, std::thread::hardware_concurrency())));
  }
  std::cout << "The end\n";
  return 0;
}
