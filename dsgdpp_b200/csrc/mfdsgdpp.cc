// mfdsgdpp.cc -- drop-in for the reference tool tools/mfdsgdpp.cc on one B200.
//
// Same options, defaults, spec strings, messages, log lines, R trace and
// .mmc/.mma/.xml files as the reference (tools/mfdsgdpp.cc:361-567,
// tools/parse.h, tools/detail/mfdsgd-args.h).  One MPI rank: the number of
// tasks d is --tasks-per-rank, and V is blocked d x 2d.  Added options:
//   --device N                   CUDA device (default 0)
//   --precision fp64|fp32|bf16   factor storage (default fp32)
//   --exec hogwild|replay        replay = the reference's sequential point
//                                order per block, FP64 only (default hogwild)
//   --launch graph|stream        epoch as one CUDA graph or 2d launches
//   --layout shuffled|col-runs|row-runs|runs   Hogwild record order in a block
// A .rm random-matrix descriptor given as --input-file (data and, with any
// --input-test-file, test matrix) or as --input-row-file (both factors) is
// generated on the device, as the reference generates it on the fly
// (mf/matrix/io/generateDistributedMatrix_impl.h:655-744).
// Invoked as `mfdsgd` (the same binary under that name) it is the drop-in for
// tools/mfdsgd.cc instead: DSGD with d x d blocks and d sub-epochs per epoch
// (mf/sgd/dsgd_impl.h), plus the --map-reduce option (on one GPU the H blocks
// stay in device memory either way, so it changes no result).
// Extension: --regularize L2(l) is accepted (the reference rejects every
// regularizer other than None, tools/mfdsgdpp.cc:165-258).
// Several ranks: started by a launcher that sets WORLD_SIZE, RANK and
// LOCAL_RANK (torchrun, for one), one process per GPU, the tool runs one job
// over the ranks as the reference does over MPI ranks: d = ranks x
// --tasks-per-rank (tools/mfdsgdpp.cc:41-42,76-77), rank r runs tasks
// r t .. (r+1) t - 1 on GPU LOCAL_RANK (unless --device is given) and the H
// blocks move between the ranks over NCCL (dsgdpp_shard_*).  Rank 0 makes the
// NCCL id and hands it over through --shard-id-file (default
// /tmp/dsgdpp-shard-<MASTER_PORT>.id); rank 0 logs and writes the outputs.
// Given --shard-id-file, a single process runs the same path (one rank).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <regex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dsgdpp.h"
#include "mmio.h"
#include "runner.h"

using namespace dsgdpp;

namespace {

struct Args {
  std::string inputMatrixFile, inputTestMatrixFile, inputRowFacFile, inputColFacFile,
      outputRowFacFile, outputColFacFile, traceFile, traceVar, sgdOrderString,
      stratumOrderString, updateString, regularizeString, lossString, decayString,
      truncateString, balanceString;
  std::string updateName, regularizeName, lossName, decayName;
  std::vector<double> updateArgs, regularizeArgs, lossArgs, truncateArgs;
  std::vector<std::string> decayArgs;
  unsigned long long epochs = 10, rank = 0;
  unsigned seed = 0;
  int tasksPerRank = 1;
  bool abs = false;
  bool mapReduce = false;  // mfdsgd --map-reduce
  double epsilon = NAN, epsDecrease = NAN, epsIncrease = NAN;
  int sgdOrder = DSGDPP_SGD_WOR, stratumOrder = DSGDPP_STRATUM_COWOR;
  // added options
  int device = 0;
  bool deviceGiven = false;
  std::string precision = "fp32", exec = "hogwild", launch = "graph", layout = "runs";
  // several ranks (WORLD_SIZE > 1)
  int world = 1, worldRank = 0, localRank = 0;
  std::string shardIdFile;
};

bool g_dsgd = false;  // running as mfdsgd

const char* kOptions[] = {
    "help", "input-file", "input-test-file", "input-row-file", "input-col-file",
    "output-row-file", "output-col-file", "trace", "trace-var", "epochs", "tasks-per-rank",
    "sgd-order", "stratum-order", "seed", "rank", "update", "regularize", "loss", "abs",
    "truncate", "decay", "balance", "device", "precision", "exec", "launch", "layout",
    "map-reduce", "shard-id-file"};

void usage() {
  std::cout << (g_dsgd ? "mfdsgd" : "mfsgdpp") << " [options]\n\nOptions:\n"
            << "  --help                 produce help message\n"
            << "  --input-file arg       filename of data matrix\n"
            << "  --input-test-file arg  filename of test matrix\n"
            << "  --input-row-file arg   filename of initial row factors\n"
            << "  --input-col-file arg   filename of initial column factors\n"
            << "  --output-row-file arg  filename of final row factors\n"
            << "  --output-col-file arg  filename of final column factors\n"
            << "  --trace arg            filename of trace [trace.R]\n"
            << "  --trace-var arg        variable name for trace [traceVar]\n"
            << "  --epochs arg           number of epochs to run [10]\n"
            << "  --tasks-per-rank arg   number of concurrent tasks per rank [1]\n"
            << "  --sgd-order arg        order of SGD steps [WOR] (e.g., \"SEQ\", \"WR\", \"WOR\")\n"
            << "  --stratum-order arg    order of strata [COWOR] (e.g., \"SEQ\", \"RSEQ\", \"WR\", "
               "\"WOR\", \"COWOR\")\n"
            << "  --seed arg             seed for random number generator (system time if not "
               "set)\n"
            << "  --rank arg             rank of factorization\n"
            << "  --update arg           SGD update function (e.g., \"Sl\", \"Nzsl\", \"GklData\")\n"
            << "  --regularize arg       SGD regularization function (e.g., \"None\", "
               "\"L2(0.05)\", \"Nzl2(0.05)\")\n"
            << "  --loss arg             loss function (e.g., \"Nzsl\", \"Nzsl_L2(0.5)\"))\n"
            << "  --abs                  if present, absolute values are taken after every SGD "
               "step\n"
            << "  --truncate arg         if present, truncatation is enabled (e.g., --truncate "
               "\"(-1000, 1000)\"\n"
            << "  --decay arg            decay function (constant, bold driver, or auto)\n"
            << "  --balance arg          Type of balancing (None, L2, Nzl2)\n"
            << "  --device arg           CUDA device [0]\n"
            << "  --precision arg        factor storage fp64|fp32|bf16 [fp32]\n"
            << "  --exec arg             hogwild|replay [hogwild]\n"
            << "  --launch arg           graph|stream [graph]\n"
            << "  --layout arg           Hogwild record order in a block:\n"
            << "                         shuffled|col-runs|row-runs|runs [runs]\n"
            << "  --shard-id-file arg    several ranks: file through which rank 0 hands the\n"
            << "                         NCCL id to the others [/tmp/dsgdpp-shard-<MASTER_PORT>.id]\n";
}

// parse::parseArg (tools/parse.h:38-61): "Name(a,b,...)" -> name + doubles
bool parse_arg(const std::string& arg, std::string& name, std::vector<std::string>& args) {
  static const std::regex re("^(.*)\\((.*)\\)$");
  std::smatch what;
  args.clear();
  if (!std::regex_match(arg, what, re)) {
    name = arg;
    return true;
  }
  name = what.str(1);
  std::string s = what.str(2);
  size_t a = 0;
  for (;;) {
    size_t c = s.find(',', a);
    args.push_back(s.substr(a, c == std::string::npos ? std::string::npos : c - a));
    if (c == std::string::npos) break;
    a = c + 1;
  }
  return true;
}

bool to_double(const std::string& t, double& v) {  // boost::lexical_cast<double>
  if (t.empty()) return false;
  char* q = nullptr;
  v = std::strtod(t.c_str(), &q);
  return q && *q == 0 && q != t.c_str();
}

void parse_doubles(const std::string& arg, std::string& name, std::vector<double>& out) {
  std::vector<std::string> a;
  parse_arg(arg, name, a);
  out.clear();
  for (size_t k = 0; k < a.size(); ++k) {
    double v;
    if (!to_double(a[k], v)) {
      std::cerr << "Invalid argument " << (k + 1) << " in " << arg << std::endl;
      std::exit(1);
    }
    out.push_back(v);
  }
}

std::string print_arg(const std::string& name, const std::vector<std::string>& a) {
  std::string s = name + "(";
  for (size_t k = 0; k < a.size(); ++k) s += (k ? "," : "") + a[k];
  return s + ")";
}

// parse::parseTruncate (tools/parse.h:114-139)
void parse_truncate(const std::string& arg, Args& args) {
  std::string name;
  std::vector<std::string> a;
  parse_arg(arg, name, a);
  double lo, hi;
  if (name.empty() && a.size() == 2 && to_double(a[0], lo) && to_double(a[1], hi)) {
    args.truncateArgs = {lo, hi};
    return;
  }
  std::cerr << "Error in argument truncate with options " << print_arg(name, a) << std::endl;
  std::cerr << "Valid options are:" << std::endl << "    (<min>,<max>)" << std::endl;
  std::exit(1);
}

// parse::parseDecay (tools/parse.h:141-235)
void parse_decay(const std::string& arg, Args& args) {
  std::string name;
  std::vector<std::string> a;
  parse_arg(arg, name, a);
  double e, x, y;
  if (name == "Const" && a.size() == 1 && to_double(a[0], e)) {
    args.decayName = "Const";
    args.epsilon = e;
    args.decayArgs = a;
    return;
  }
  if (name == "Auto" && a.size() == 3 && to_double(a[0], e)) {
    args.decayName = "Auto";
    args.decayArgs = a;
    return;
  }
  if (name == "BoldDriver" && a.size() == 1 && to_double(a[0], e)) {
    args.decayName = "BoldDriver";
    args.epsilon = e;
    args.epsDecrease = NAN;
    args.epsIncrease = NAN;
    args.decayArgs = a;
    return;
  }
  if (name == "BoldDriver" && a.size() == 3 && to_double(a[0], e) && to_double(a[1], x) &&
      to_double(a[2], y)) {
    args.decayName = "BoldDriver";
    args.epsilon = e;
    args.epsDecrease = x;
    args.epsIncrease = y;
    args.decayArgs = a;
    return;
  }
  if (name == "Sequential" && (a.size() == 1 || a.size() == 3) && to_double(a[0], e)) {
    args.decayName = "Sequential";
    args.decayArgs = a;
    return;
  }
  std::cerr << "Error in argument 'decay': Unknown or invalid loss '" << print_arg(name, a) << "'"
            << std::endl;
  std::cerr << "Valid choices are: " << std::endl
            << "    Const(<epsilon>)" << std::endl
            << "    Auto(<epsilon>,<tries>,<input-sample-matrix>)" << std::endl
            << "    BoldDriver(<epsilon>)" << std::endl
            << "    BoldDriver(<epsilon>,<epsDecrease>,<epsIncrease>)" << std::endl
            << "    Sequential(<epsilon>)" << std::endl
            << "    Sequential(<epsilon>,<alpha>,<A>)" << std::endl;
  std::exit(1);
}

struct Job {
  int update, regularize, loss;
  double update_lambda = 0, regularize_lambda = 0, loss_lambda = 0;
};

// runArgs (tools/mfdsgdpp.cc:162-359): the valid (update, regularize, loss)
// combinations and their argument counts.
bool resolve(const Args& a, Job& job) {
  auto arity = [&](const std::vector<double>& v, size_t n, const std::string& s) {
    if (v.size() != n) {
      std::cout << "Invalid number of arguments in " << s << std::endl;
      return false;
    }
    return true;
  };
  if (!a.abs) {
    const bool reg_none = a.regularizeName == "None";
    const bool reg_l2 = a.regularizeName == "L2";  // extension
    if (reg_none || reg_l2) {
      if (reg_l2 && !arity(a.regularizeArgs, 1, a.regularizeString)) return false;
      if (reg_none && !arity(a.regularizeArgs, 0, a.regularizeString)) return false;
      job.regularize = reg_l2 ? DSGDPP_REGULARIZE_L2 : DSGDPP_REGULARIZE_NONE;
      job.regularize_lambda = reg_l2 ? a.regularizeArgs[0] : 0;
      if (a.updateName == "Nzsl" && a.lossName == "Nzsl") {
        if (!arity(a.updateArgs, 0, a.updateString) || !arity(a.lossArgs, 0, a.lossString))
          return false;
        job.update = DSGDPP_UPDATE_NZSL;
        job.loss = DSGDPP_LOSS_NZSL;
        return true;
      }
      if (a.updateName == "Nzsl_L2" && a.lossName == "Nzsl_L2") {
        if (!arity(a.updateArgs, 1, a.updateString) || !arity(a.lossArgs, 1, a.lossString))
          return false;
        job.update = DSGDPP_UPDATE_NZSL_L2;
        job.update_lambda = a.updateArgs[0];
        job.loss = DSGDPP_LOSS_NZSL_L2;
        job.loss_lambda = a.lossArgs[0];
        return true;
      }
      if (a.updateName == "Nzsl_Nzl2" && a.lossName == "Nzsl_Nzl2") {
        if (!arity(a.updateArgs, 1, a.updateString) || !arity(a.lossArgs, 1, a.lossString))
          return false;
        job.update = DSGDPP_UPDATE_NZSL_NZL2;
        job.update_lambda = a.updateArgs[0];
        job.loss = DSGDPP_LOSS_NZSL_NZL2;
        job.loss_lambda = a.lossArgs[0];
        return true;
      }
    }
  }
  std::cerr << "Invalid combination of update, regularize, and loss arguments" << std::endl;
  std::cout << "Valid combinations are:" << std::endl;
  std::cout << "\tNzsl / None / Nzsl" << std::endl;
  std::cout << "\tNzsl / L2 / Nzsl_L2" << std::endl;
  std::cout << "\tNzsl_Nzl2 / None / Nzsl_Nzl2" << std::endl;
  return false;
}

std::string blocks_list(uint64_t b1, uint64_t b2) {
  std::string s;
  for (uint64_t i = 0; i < b1; ++i)
    for (uint64_t j = 0; j < b2; ++j) s += "(" + std::to_string(i) + "," + std::to_string(j) + ") ";
  return s;
}

// Rank 0 makes the NCCL id and publishes it in `path` (written under another
// name, then renamed); the other ranks wait for the file, at most `limit_s`.
std::vector<char> exchange_shard_id(const Args& args, double limit_s = 300) {
  std::vector<char> id(DSGDPP_SHARD_ID_BYTES);
  const std::string& path = args.shardIdFile;
  if (args.worldRank == 0) {
    const int rc = dsgdpp_shard_unique_id(id.data());
    if (rc != DSGDPP_OK) throw CallError(rc, "dsgdpp_shard_unique_id: NCCL is not available");
    const std::string tmp = path + ".tmp";
    {
      std::ofstream f(tmp, std::ios::binary | std::ios::trunc);
      f.write(id.data(), (std::streamsize)id.size());
      if (!f) throw std::runtime_error("cannot write " + tmp);
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0)
      throw std::runtime_error("cannot rename " + tmp + " to " + path);
    return id;
  }
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    std::ifstream f(path, std::ios::binary);
    if (f && f.read(id.data(), (std::streamsize)id.size()) && f.gcount() == (std::streamsize)id.size())
      return id;
    if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > limit_s)
      throw std::runtime_error("no NCCL id from rank 0 in " + path + " within " +
                               std::to_string((int)limit_s) + " s");
    std::this_thread::sleep_for(std::chrono::milliseconds(20));
  }
}

int run(Args& args, const Job& job) {
  // d = ranks x tasks per rank (tools/mfdsgdpp.cc:41-42,76-77)
  const uint32_t d = (uint32_t)(args.tasksPerRank * args.world);
  const bool sharded = args.world > 1 || !args.shardIdFile.empty();
  const uint32_t nb2 = g_dsgd ? d : 2 * d;  // column blocks: d x d (DSGD) or d x 2d (DSGD++)
  if (args.decayName != "BoldDriver" && args.decayName != "Const") {
    std::cerr << "not implemented: decay" << std::endl;  // rg::NotImplementedException
    return 1;
  }
  auto t0 = std::chrono::steady_clock::now();
  auto load_sparse = [&](const std::string& f) {
    BlockedDescriptor desc;
    if (!ends_with(f, ".xml")) {
      Log::info("mf", "File '" + f + "' is not blocked; it will be blocked automatically");
      Log::info("mf", "Constructing blocks " + blocks_list(d, nb2) + " of '" + f + "'");
    }
    Coo m = read_sparse(f, &desc);
    if (ends_with(f, ".xml")) {
      // the descriptor's blocking must be the job's default blocking, d x 2d
      // (checkBlockingDsgdPp, mf/sgd/dsgdpp-factorization.h:21-33) or d x d
      std::vector<uint64_t> o1(d), o2(nb2);
      dsgdpp_block_offsets(desc.size1, d, o1.data());
      dsgdpp_block_offsets(desc.size2, nb2, o2.data());
      if (desc.blocks1 != d || desc.blocks2 != nb2 || desc.offsets1 != o1 || desc.offsets2 != o2)
        throw std::invalid_argument("blocking of " + f + " does not match the d x " +
                                    (g_dsgd ? std::string("d") : std::string("2d")) +
                                    " job blocking");
    }
    return m;
  };
  // .rm descriptors: matrices generated on the device instead of read
  // (getDataMatrices / getFactors, generateDistributedMatrix_impl.h:655-744)
  using RmPtr = std::unique_ptr<dsgdpp_rm, void (*)(dsgdpp_rm*)>;
  auto load_rm = [](const std::string& f) {
    dsgdpp_rm* h = nullptr;
    if (dsgdpp_rm_load(f.c_str(), &h) != DSGDPP_OK) throw std::invalid_argument(dsgdpp_rm_error());
    RmPtr p(h, dsgdpp_rm_destroy);
    return p;
  };
  RmPtr rmV(nullptr, dsgdpp_rm_destroy), rmF(nullptr, dsgdpp_rm_destroy);
  uint64_t info_v[9] = {0}, info_f[9] = {0};
  Coo V, T;
  const bool has_test = !args.inputTestMatrixFile.empty();
  uint64_t Vm, Vn, Vnnz, Tm = 0, Tn = 0, Tnnz = 0;
  if (ends_with(args.inputMatrixFile, ".rm")) {
    rmV = load_rm(args.inputMatrixFile);
    dsgdpp_rm_info(rmV.get(), info_v);
    Log::info("mf", "generating data matrices on the fly...");
    if (info_v[7] == 0 && info_v[5] == 0)
      throw std::invalid_argument(args.inputMatrixFile + " holds no data matrix (nnz or nnzTest is 0)");
    Vm = Tm = info_v[0];
    Vn = Tn = info_v[1];
    Vnnz = info_v[7];
    Tnnz = info_v[8];  // the test matrix comes from the same descriptor
  } else {
    V = load_sparse(args.inputMatrixFile);
    Vm = V.size1; Vn = V.size2; Vnnz = V.vals.size();
    if (has_test) {
      T = load_sparse(args.inputTestMatrixFile);
      Tm = T.size1; Tn = T.size2; Tnnz = T.vals.size();
    }
  }
  if (has_test)
    Log::info("mf", "Test matrix: " + std::to_string(Tm) + " x " + std::to_string(Tn) + ", " +
                        std::to_string(Tnnz) + " nonzeros, " + std::to_string(d) + " x " +
                        std::to_string(nb2) + " blocks");
  Log::info("mf", "Data matrix: " + std::to_string(Vm) + " x " + std::to_string(Vn) + ", " +
                      std::to_string(Vnnz) + " nonzeros, " + std::to_string(d) + " x " +
                      std::to_string(nb2) + " blocks");
  Dense Wf, Hf;
  if (ends_with(args.inputRowFacFile, ".rm")) {  // both factors from this one descriptor
    Log::info("mf", "generating factors on the fly...");
    rmF = load_rm(args.inputRowFacFile);
    dsgdpp_rm_info(rmF.get(), info_f);
    Wf.size1 = info_f[0]; Wf.size2 = info_f[2];
    Hf.size1 = info_f[2]; Hf.size2 = info_f[1];
  } else {
    // .mma, or the .xml of .mma blocks that mfdblock writes for a dense matrix
    for (const std::string* f : {&args.inputRowFacFile, &args.inputColFacFile})
      if (!ends_with(*f, ".xml"))
        Log::info("mf", "File '" + *f + "' is not blocked; it will be blocked automatically");
    Wf = read_dense(args.inputRowFacFile);
    Hf = read_dense(args.inputColFacFile);
  }
  Log::info("mf", "Row factor matrix: " + std::to_string(Wf.size1) + " x " +
                      std::to_string(Wf.size2) + ", " + std::to_string(d) + " x 1 blocks");
  Log::info("mf", "Column factor matrix: " + std::to_string(Hf.size1) + " x " +
                      std::to_string(Hf.size2) + ", 1 x " + std::to_string(nb2) + " blocks");
  // conformity (mf/factorization.h:27-33)
  if (Wf.size1 != Vm || Hf.size2 != Vn || Wf.size2 != Hf.size1 ||
      (has_test && (Tm != Vm || Tn != Vn)))
    throw std::invalid_argument("factor and data matrices do not conform");
  if (Wf.size2 != args.rank)
    Log::info("main", "Warning: --rank differs from the factor files; using " +
                          std::to_string(Wf.size2));
  const uint64_t m = Vm, n = Vn, r = Wf.size2;
  // W: m x r column-major in the file -> row-major; H: r x n column-major = n x r rows
  std::vector<double> W, H;
  if (!rmF) {
    W.resize(m * r);
    H.resize(n * r);
    for (uint64_t i = 0; i < m; ++i)
      for (uint64_t z = 0; z < r; ++z) W[i * r + z] = Wf.colmajor[z * m + i];
    for (uint64_t j = 0; j < n; ++j)
      for (uint64_t z = 0; z < r; ++z) H[j * r + z] = Hf.colmajor[j * r + z];
  }
  auto t1 = std::chrono::steady_clock::now();
  Log::info("main", "Total time for loading matrices: " +
                        fmt_secs((double)std::chrono::duration_cast<std::chrono::nanoseconds>(t1 - t0).count()));

  dsgdpp_config cfg;
  dsgdpp_config_init(&cfg);
  cfg.m = m;
  cfg.n = n;
  cfg.rank = (uint32_t)r;
  cfg.d = d;
  cfg.method = g_dsgd ? DSGDPP_METHOD_DSGD : DSGDPP_METHOD_DSGDPP;
  cfg.precision = args.precision == "fp64" ? DSGDPP_FP64 : args.precision == "bf16" ? DSGDPP_BF16 : DSGDPP_FP32;
  cfg.exec = args.exec == "replay" ? DSGDPP_EXEC_REPLAY : DSGDPP_EXEC_HOGWILD;
  cfg.launch = args.launch == "stream" ? DSGDPP_LAUNCH_STREAM : DSGDPP_LAUNCH_GRAPH;
  cfg.layout = args.layout == "col-runs"   ? DSGDPP_LAYOUT_COL_RUNS
               : args.layout == "row-runs" ? DSGDPP_LAYOUT_ROW_RUNS
               : args.layout == "runs"     ? DSGDPP_LAYOUT_RUNS
                                           : DSGDPP_LAYOUT_SHUFFLED;
  cfg.update = job.update;
  cfg.update_lambda = job.update_lambda;
  cfg.regularize = job.regularize;
  cfg.regularize_lambda = job.regularize_lambda;
  cfg.loss = job.loss;
  cfg.loss_lambda = job.loss_lambda;
  if (!std::isnan(args.truncateArgs[0]) && !std::isnan(args.truncateArgs[1])) {
    cfg.truncate = 1;
    cfg.truncate_min = args.truncateArgs[0];
    cfg.truncate_max = args.truncateArgs[1];
  }
  cfg.sgd_order = args.sgdOrder;
  cfg.stratum_order = args.stratumOrder;
  cfg.device = args.device;
  if (sharded && cfg.launch == DSGDPP_LAUNCH_GRAPH)
    cfg.launch = DSGDPP_LAUNCH_STREAM;  // a sharded epoch runs one sub-epoch at a time
  dsgdpp_ctx* ctx = nullptr;
  int rc = dsgdpp_create(&cfg, &ctx);
  if (rc != DSGDPP_OK) throw CallError(rc, std::string("dsgdpp_create: ") + dsgdpp_create_error());
  struct Guard {
    dsgdpp_ctx* c;
    ~Guard() { dsgdpp_destroy(c); }
  } guard{ctx};
  if (sharded) {
    // this rank's tasks' rows of V and of the test matrix; the update weights
    // count the whole matrix; W is zero outside this rank's rows
    if (rmV) {
      for (int which : {DSGDPP_TRAIN, DSGDPP_TEST}) {
        if (which == DSGDPP_TEST && !has_test) continue;
        Coo& M = which == DSGDPP_TRAIN ? V : T;
        const uint64_t cnt = info_v[which == DSGDPP_TRAIN ? 7 : 8];
        M.size1 = m;
        M.size2 = n;
        M.rows.resize(cnt);
        M.cols.resize(cnt);
        M.vals.resize(cnt);
        check(ctx, dsgdpp_rm_generate(rmV.get(), which, cfg.device, M.rows.data(),
                                      M.cols.data(), M.vals.data()), "rm_generate");
      }
    }
    if (rmF) {
      W.resize(m * r);
      H.resize(n * r);
      check(ctx, dsgdpp_rm_generate_factors(rmF.get(), cfg.device, W.data(), H.data()),
            "rm_generate_factors");
    }
    std::vector<uint64_t> off1(d + 1);
    dsgdpp_block_offsets(m, d, off1.data());
    off1[d] = m;
    const uint32_t t = (uint32_t)args.tasksPerRank, first = (uint32_t)args.worldRank * t;
    const uint64_t lo = off1[first], hi = off1[first + t];
    std::vector<uint64_t> n1(m, 0), n2(n, 0);
    for (size_t k = 0; k < V.vals.size(); ++k) {
      n1[V.rows[k]]++;
      n2[V.cols[k]]++;
    }
    auto own = [&](const Coo& M) {
      Coo o;
      for (size_t k = 0; k < M.vals.size(); ++k)
        if (M.rows[k] >= lo && M.rows[k] < hi) {
          o.rows.push_back(M.rows[k]);
          o.cols.push_back(M.cols[k]);
          o.vals.push_back(M.vals[k]);
        }
      return o;
    };
    check(ctx, dsgdpp_set_tasks(ctx, first, t), "set_tasks");
    const Coo Vr = own(V);
    check(ctx, dsgdpp_set_matrix(ctx, DSGDPP_TRAIN, Vr.vals.size(), Vr.rows.data(),
                                 Vr.cols.data(), Vr.vals.data()), "set_matrix");
    if (has_test) {
      const Coo Tr = own(T);
      check(ctx, dsgdpp_set_matrix(ctx, DSGDPP_TEST, Tr.vals.size(), Tr.rows.data(),
                                   Tr.cols.data(), Tr.vals.data()), "set_matrix");
    }
    check(ctx, dsgdpp_set_counts(ctx, n1.data(), n2.data()), "set_counts");
    std::vector<double> Wr(m * r, 0.0);
    std::copy(W.begin() + lo * r, W.begin() + hi * r, Wr.begin() + lo * r);
    check(ctx, dsgdpp_set_factors(ctx, Wr.data(), H.data()), "set_factors");
  } else if (rmV) {
    check(ctx, dsgdpp_set_matrix_rm(ctx, DSGDPP_TRAIN, rmV.get()), "set_matrix_rm");
    if (has_test) check(ctx, dsgdpp_set_matrix_rm(ctx, DSGDPP_TEST, rmV.get()), "set_matrix_rm");
  } else {
    check(ctx, dsgdpp_set_matrix(ctx, DSGDPP_TRAIN, V.vals.size(), V.rows.data(),
                                 V.cols.data(), V.vals.data()), "set_matrix");
    if (has_test)
      check(ctx, dsgdpp_set_matrix(ctx, DSGDPP_TEST, T.vals.size(), T.rows.data(),
                                   T.cols.data(), T.vals.data()), "set_matrix");
  }
  if (sharded) {
  } else if (rmF) {
    check(ctx, dsgdpp_set_factors_rm(ctx, rmF.get()), "set_factors_rm");
  } else {
    check(ctx, dsgdpp_set_factors(ctx, W.data(), H.data()), "set_factors");
  }
  check(ctx, dsgdpp_seed(ctx, args.seed), "seed");
  std::unique_ptr<dsgdpp_shard, void (*)(dsgdpp_shard*)> shard(nullptr, dsgdpp_shard_destroy);
  if (sharded) {
    const std::vector<char> id = exchange_shard_id(args);
    dsgdpp_shard* sh = nullptr;
    check(ctx, dsgdpp_shard_create_nccl(ctx, args.worldRank, args.world, id.data(), &sh),
          "dsgdpp_shard_create_nccl");
    shard.reset(sh);
    if (args.worldRank == 0) std::remove(args.shardIdFile.c_str());  // every rank has joined
  }

  Trace trace;  // Args::createTraceFields (tools/detail/mfdsgd-args.h:53-63)
  trace.add_field("update", args.updateString);
  trace.add_field("regularize", args.regularizeString);
  trace.add_field("rank", (double)args.rank);
  trace.add_field("input_file", args.inputMatrixFile);
  trace.add_field("sample_matrix", "");
  trace.add_field("nodes", (double)args.world);
  trace.add_field("threads", (double)args.tasksPerRank);
  trace.add_field("barrier", "false");

  Decay decay;
  decay.kind = args.decayName == "Const" ? DSGDPP_DECAY_CONST : DSGDPP_DECAY_BOLDDRIVER;
  decay.eps = args.epsilon;
  if (!std::isnan(args.epsDecrease) || !std::isnan(args.epsIncrease)) {
    decay.decrease = args.epsDecrease;
    decay.increase = args.epsIncrease;
  }
  if (has_test) Log::info("main", "Using NzslLoss for test data");
  Log::info("mf", std::string(g_dsgd ? "Starting DSGD" : "Starting DSGD++") + " on " +
                      std::string(args.exec) + " " + args.precision +
                      (sharded ? " (B200, " + std::to_string(args.world) + " ranks, one GPU each)"
                               : std::string(" (B200, one GPU)")));
  if (g_dsgd)  // mf/sgd/dsgd_impl.h:56-60
    Log::info("mf", args.mapReduce ? "Using slow MapReduce-style implementation"
                                   : "Using fast DSGD+ implementation");
  static const char* kStrata[] = {"SEQ", "RSEQ", "WR", "WOR", "COWOR"};
  static const char* kPoints[] = {"SEQ", "WR", "WOR"};
  Log::info("mf", std::string("Using ") + kStrata[args.stratumOrder] + " order for selecting strata");
  Log::info("mf", std::string("Using ") + kPoints[args.sgdOrder] +
                      " order for selecting training points");
  auto r0 = std::chrono::steady_clock::now();
  if (shard)
    shard_runner(shard.get(), args.epochs, decay, trace, has_test);
  else
    default_runner(ctx, args.epochs, decay, trace, has_test);
  auto r1 = std::chrono::steady_clock::now();
  Log::info("mf", g_dsgd ? "Finished DSGD" : "Finished DSGD++");
  Log::info("main", "Total time: " +
                        fmt_secs((double)std::chrono::duration_cast<std::chrono::nanoseconds>(r1 - r0).count()));

  const bool writer = args.worldRank == 0;  // rank 0 writes the outputs
  if (shard && (!args.outputRowFacFile.empty() || !args.outputColFacFile.empty()))
    check_shard(shard.get(), dsgdpp_shard_gather_w(shard.get()), "shard gather W");
  if (!writer) return 0;
  if (!args.traceFile.empty()) {
    Log::info("main", "Writing trace to " + args.traceFile);
    std::ofstream f(args.traceFile);
    f << trace.to_r(args.traceVar);
  }
  if (!args.outputRowFacFile.empty() || !args.outputColFacFile.empty()) {
    W.resize(m * r);  // empty when the factors were generated from a descriptor
    H.resize(n * r);
    check(ctx, dsgdpp_get_factors(ctx, W.data(), H.data()), "get_factors");
  }
  if (!args.outputRowFacFile.empty()) {
    Log::info("main", "Writing row factors to " + args.outputRowFacFile);
    Dense o;
    o.size1 = m;
    o.size2 = r;
    o.colmajor.resize(m * r);
    for (uint64_t i = 0; i < m; ++i)
      for (uint64_t z = 0; z < r; ++z) o.colmajor[z * m + i] = W[i * r + z];
    write_mm_array(args.outputRowFacFile, o);
  }
  if (!args.outputColFacFile.empty()) {
    Log::info("main", "Writing column factors to " + args.outputColFacFile);
    Dense o;
    o.size1 = r;
    o.size2 = n;
    o.colmajor = H;  // column j of H is contiguous
    write_mm_array(args.outputColFacFile, o);
  }
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  {
    const std::string self = argc > 0 ? std::string(argv[0]) : std::string();
    const size_t slash = self.find_last_of('/');
    g_dsgd = self.substr(slash == std::string::npos ? 0 : slash + 1) == "mfdsgd";
  }
  Args args;
  std::map<std::string, std::string> vm;
  std::vector<std::string> positional;
  const std::vector<std::string> flags(std::begin(kOptions), std::end(kOptions));
  for (int k = 1; k < argc; ++k) {
    std::string a = argv[k];
    if (a.rfind("--", 0) == 0) {
      std::string key = a.substr(2), val;
      size_t eq = key.find('=');
      if (eq != std::string::npos) {
        val = key.substr(eq + 1);
        key = key.substr(0, eq);
      } else if (key != "help" && key != "abs") {
        if (k + 1 >= argc) {
          std::cerr << "the required argument for option '--" << key << "' is missing" << std::endl;
          return 1;
        }
        val = argv[++k];
      }
      if (std::find(flags.begin(), flags.end(), key) == flags.end() ||
          (key == "map-reduce" && !g_dsgd)) {
        std::cerr << "unrecognised option '--" << key << "'" << std::endl;
        return 1;
      }
      vm[key] = val;
    } else {
      positional.push_back(a);
    }
  }
  const char* pos_names[] = {"input-file", "input-test-file", "input-row-file", "input-col-file",
                             "output-row-file", "output-col-file"};
  for (size_t k = 0; k < positional.size() && k < 6; ++k)
    if (!vm.count(pos_names[k])) vm[pos_names[k]] = positional[k];

  const char* required[] = {"input-file", "input-row-file", "input-col-file", "update",
                            "regularize", "loss", "rank", "decay"};
  bool missing = vm.count("help") > 0;
  for (auto r : required) missing = missing || !vm.count(r);
  if (missing) {
    std::cerr << "Error: Options input-file, input-row-file, input-col-file, update, regularize, "
                 "loss, rank, and decay have to be present"
              << std::endl;
    usage();
    return 1;
  }
  auto get = [&](const char* k, const std::string& dflt) { return vm.count(k) ? vm[k] : dflt; };
  args.inputMatrixFile = vm["input-file"];
  args.inputTestMatrixFile = get("input-test-file", "");
  args.inputRowFacFile = vm["input-row-file"];
  args.inputColFacFile = vm["input-col-file"];
  args.outputRowFacFile = get("output-row-file", "");
  args.outputColFacFile = get("output-col-file", "");
  args.traceFile = get("trace", "");
  args.traceVar = get("trace-var", "trace");
  try {
    args.seed = vm.count("seed") ? (unsigned)std::stoul(vm["seed"]) : (unsigned)std::time(nullptr);
    args.epochs = vm.count("epochs") ? std::stoull(vm["epochs"]) : 10;
    args.tasksPerRank = vm.count("tasks-per-rank") ? std::stoi(vm["tasks-per-rank"]) : 1;
    args.rank = std::stoull(vm["rank"]);
    args.deviceGiven = vm.count("device") > 0;
    args.device = args.deviceGiven ? std::stoi(vm["device"]) : 0;
    auto env_int = [](const char* k, int dflt) {
      const char* v = std::getenv(k);
      return v && *v ? std::stoi(v) : dflt;
    };
    args.world = env_int("WORLD_SIZE", 1);
    args.worldRank = env_int("RANK", 0);
    args.localRank = env_int("LOCAL_RANK", 0);
  } catch (const std::exception&) {
    std::cerr << "invalid numeric option value" << std::endl;
    return 1;
  }
  args.sgdOrderString = get("sgd-order", "WOR");
  args.stratumOrderString = get("stratum-order", "COWOR");
  args.updateString = vm["update"];
  args.regularizeString = vm["regularize"];
  args.lossString = vm["loss"];
  args.decayString = vm["decay"];
  args.balanceString = get("balance", "None");
  if (args.world < 1 || args.worldRank < 0 || args.worldRank >= args.world) {
    std::cerr << "invalid WORLD_SIZE / RANK" << std::endl;
    return 1;
  }
  if (args.world > 1 || vm.count("shard-id-file")) {
    if (!args.deviceGiven) args.device = args.localRank;
    const char* port = std::getenv("MASTER_PORT");
    args.shardIdFile = get("shard-id-file", std::string("/tmp/dsgdpp-shard-") +
                                                (port && *port ? port : "0") + ".id");
    Log::quiet() = args.worldRank != 0;
  }
  args.precision = get("precision", "fp32");
  args.exec = get("exec", "hogwild");
  args.launch = get("launch", "graph");
  args.layout = get("layout", "runs");
  if (args.layout != "shuffled" && args.layout != "col-runs" && args.layout != "row-runs" &&
      args.layout != "runs") {
    std::cerr << "unknown --layout " << args.layout << std::endl;
    return 1;
  }

  Log::info("main", "Input");
  Log::info("main", "    Input file: " + args.inputMatrixFile);
  Log::info("main", "    Input test file: " +
                        (args.inputTestMatrixFile.empty() ? std::string("Disabled") : args.inputTestMatrixFile));
  Log::info("main", "    Input row factors: " + args.inputRowFacFile);
  Log::info("main", "    Input column factors: " + args.inputColFacFile);
  Log::info("main", "Output");
  Log::info("main", "    Output row factors: " +
                        (args.outputRowFacFile.empty() ? std::string("Disabled") : args.outputRowFacFile));
  Log::info("main", "    Output column factors: " +
                        (args.outputColFacFile.empty() ? std::string("Disabled") : args.outputColFacFile));
  Log::info("main", args.traceFile.empty() ? std::string("    Trace: Disabled")
                                           : "    Trace: " + args.traceFile + " (" + args.traceVar + ")");
  Log::info("main", "Parallelization");
  Log::info("main", "    MPI ranks: " + std::to_string(args.world));
  Log::info("main", "    Tasks per rank: " + std::to_string(args.tasksPerRank));
  Log::info("main", g_dsgd ? "DSGD options" : "DSGD++ options");
  Log::info("main", "    Seed: " + std::to_string(args.seed));
  Log::info("main", "    Epochs: " + std::to_string(args.epochs));
  Log::info("main", "    Factorization rank: " + std::to_string(args.rank));
  Log::info("main", "    Update function: " + args.updateString);
  Log::info("main", "    Regularize function: " + args.regularizeString);
  Log::info("main", "    Loss function: " + args.lossString);
  Log::info("main", "    Decay: " + args.decayString);

  if (args.balanceString == "None") {
    Log::info("main", "    Balancing: Disabled");
  } else if (args.balanceString == "L2" || args.balanceString == "NZL2") {
    std::cerr << "Balancing " << args.balanceString << " is not supported on the GPU path" << std::endl;
    return 1;
  } else {
    std::cerr << "Invalid arguments for balance; expected \"None\", \"L2\" or \"Nzl2\"" << std::endl;
    return 1;
  }
  args.abs = vm.count("abs") > 0;
  Log::info("main", args.abs ? "    Absolute function: Enabled" : "    Absolute function: Disabled");
  if (!vm.count("truncate")) {
    args.truncateArgs = {NAN, NAN};
    Log::info("main", "    Truncation: Disabled");
  } else {
    parse_truncate(vm["truncate"], args);
    Log::info("main", "    Truncation: (" + fmt_g(args.truncateArgs[0]) + "," +
                          fmt_g(args.truncateArgs[1]) + ")");
  }
  if (args.sgdOrderString == "SEQ") args.sgdOrder = DSGDPP_SGD_SEQ;
  else if (args.sgdOrderString == "WR") args.sgdOrder = DSGDPP_SGD_WR;
  else if (args.sgdOrderString == "WOR") args.sgdOrder = DSGDPP_SGD_WOR;
  else {
    std::cerr << "Invalid arguments for sgdOrder; expected \"SEQ\", \"WR\" or \"WOR\"" << std::endl;
    return 1;
  }
  Log::info("main", "    SGD step sequence: " + args.sgdOrderString);
  const char* strata[] = {"SEQ", "RSEQ", "WR", "WOR", "COWOR"};
  int so = -1;
  for (int k = 0; k < 5; ++k)
    if (args.stratumOrderString == strata[k]) so = k;
  if (so < 0) {
    std::cerr << "Invalid arguments for stratumOrder; expected \"SEQ\", \"RSEQ\", \"WR\", \"WOR\" "
                 "or \"COWOR\""
              << std::endl;
    return 1;
  }
  args.stratumOrder = so;
  Log::info("main", "    DSGD stratum sequence: " + args.stratumOrderString);
  if (g_dsgd) {  // tools/mfdsgd.cc:63,108,211 (boost bool syntax)
    const std::string mr = vm.count("map-reduce") ? vm["map-reduce"] : "0";
    if (mr == "1" || mr == "true" || mr == "yes" || mr == "on") {
      args.mapReduce = true;
    } else if (mr == "0" || mr == "false" || mr == "no" || mr == "off") {
      args.mapReduce = false;
    } else {
      std::cerr << "the argument ('" << mr << "') for option '--map-reduce' is invalid" << std::endl;
      return 1;
    }
    Log::info("main", std::string("    Slow MapReduce implementation: ") +
                          (args.mapReduce ? "1" : "0"));
  }

  parse_doubles(args.updateString, args.updateName, args.updateArgs);
  parse_doubles(args.regularizeString, args.regularizeName, args.regularizeArgs);
  parse_doubles(args.lossString, args.lossName, args.lossArgs);
  parse_decay(args.decayString, args);

  Job job{};
  if (!resolve(args, job)) return 1;
  if (args.tasksPerRank < 1) {
    std::cerr << "tasks-per-rank must be positive" << std::endl;
    return 1;
  }
  try {
    return run(args, job);
  } catch (const MmError& e) {
    std::cerr << "I/O error: " << e.what() << std::endl;
  } catch (const CallError& e) {
    std::cerr << "error: " << e.what() << std::endl;
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
  }
  return 1;
}
