// bin/* drivers with the reference programs' argument order and result CSV.
//
//   TrimCDP      2   <path> <data> <k> <s> <e>        (code/TrimCDP/src/main.cpp:14-16)
//   D-TrimCDP    2   <path> <data> <k> <D> <s> <e>    (code/D-TrimCDP/src/main.cpp:18-20)
//   TrimCDP-WB   <x> <path> <data> <k> <s> <e>        (code/TrimCDP-WB/src/GSTnonHop.cu:195-196)
//   D-TrimCDP-WB <x> <path> <data> <k> <D> <s> <e>    (code/D-TrimCDP-WB/src/GPUHop.cu:98-99)
//
// <s>..<e> is an inclusive 0-based range of lines of <path><data><k>.csv.  The
// text-graph programs read <path><data>.in, the -WB programs the int64 binary
// CSR <path><data>_{beg_pos,csr,weight}.bin; all read <path><data>.g.  Each
// writes <path>result/exp_<TAG>_<data>_T<k>[_D<D>]_<s>-<e>.csv with the
// reference's header (exp_GPU_nonHop.h:83-85, exp_GPU_Hop.h:75-77,
// GSTnonHop.cu:264-266, GPUHop.cu:157-159).  Columns: query index, the group
// ids, per-query device time (s), cost, memory (table entries of the touched
// vertices), counts (vertices that held a finite state), process_num (states
// expanded).  An infeasible query prints the cost its reference program
// prints: 0 for TrimCDP (DPQ.cu:571-575), 100000 for the others.
//
// The queries of the range are solved as one batch; GST_ONE_AT_A_TIME=1
// solves them one call at a time like the reference.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gst_b200.h"

#ifndef GST_PROGRAM
#define GST_PROGRAM "TrimCDP"
#endif

static int die(const char* what) {
  std::fprintf(stderr, "%s: %s (%s)\n", GST_PROGRAM, what, gst_last_error());
  return 1;
}

int main(int argc, char** argv) {
  const std::string prog = GST_PROGRAM;
  const bool hop = prog.rfind("D-", 0) == 0;
  const bool wb = prog.find("-WB") != std::string::npos;
  const int need = hop ? 8 : 7;
  if (argc < need) {
    std::fprintf(stderr, "usage: %s <mode> <path> <data> <k>%s <start> <end>\n", GST_PROGRAM,
                 hop ? " <D>" : "");
    return 2;
  }
  if (!wb && std::atoi(argv[1]) != 2) {  // the reference programs run only mode 2
    std::fprintf(stderr, "%s: mode %s does nothing (the reference runs mode 2)\n", GST_PROGRAM, argv[1]);
    return 0;
  }
  const std::string path = argv[2], data = argv[3];
  const int k = std::atoi(argv[4]);
  const int D = hop ? std::atoi(argv[5]) : -1;
  const int s = std::atoi(argv[hop ? 6 : 5]), e = std::atoi(argv[hop ? 7 : 6]);

  gst_csr g{};
  gst_status st = wb ? gst_read_binary_csr((path + data + "_beg_pos.bin").c_str(),
                                           (path + data + "_csr.bin").c_str(),
                                           (path + data + "_weight.bin").c_str(), &g)
                     : gst_read_input_graph((path + data + ".in").c_str(), &g);
  if (st != GST_OK) return die("graph");
  gst_groups gr{};
  if (gst_read_groups((path + data + ".g").c_str(), &gr) != GST_OK) return die("groups");
  gst_queries qs{};
  if (gst_read_queries((path + data + std::to_string(k) + ".csv").c_str(), &qs) != GST_OK)
    return die("queries");
  if (s < 0 || e < s || e >= qs.n) {
    std::fprintf(stderr, "%s: query range %d-%d outside 0-%lld\n", GST_PROGRAM, s, e, (long long)qs.n - 1);
    return 1;
  }
  gst_engine* eng = nullptr;
  gst_engine_config cfg{};
  if (const char* dev = std::getenv("GST_DEVICE")) cfg.device = std::atoi(dev);
  if (gst_engine_create(&cfg, &eng) != GST_OK) return die("engine");
  if (gst_engine_load_graph(eng, g.V, g.rowptr, g.col, g.w) != GST_OK) return die("load graph");
  if (gst_engine_load_groups(eng, gr.n, gr.ptr, gr.members) != GST_OK) return die("load groups");

  const int n = e - s + 1;
  std::vector<gst_result> res(n);
  std::vector<gst_status> sts(n, GST_OK);
  const char* one = std::getenv("GST_ONE_AT_A_TIME");
  if (one && std::atoi(one) == 1) {
    for (int i = 0; i < n; ++i) {
      const int64_t b = qs.ptr[s + i];
      sts[i] = gst_solve(eng, qs.ids + b, (int)(qs.ptr[s + i + 1] - b), D, &res[i]);
    }
  } else {
    std::vector<int64_t> ptr(n + 1);
    for (int i = 0; i <= n; ++i) ptr[i] = qs.ptr[s + i] - qs.ptr[s];
    std::vector<int32_t> Ds(n, D);
    if (gst_solve_batch(eng, n, ptr.data(), qs.ids + qs.ptr[s], Ds.data(), res.data(), sts.data()) != GST_OK)
      return die("solve");
  }

  std::string tag = std::string(wb ? "GPU2_" : "GPU1_") + (hop ? "Hop" : "nonHop");
  std::string fn = path + "result/exp_" + tag + "_" + data + "_T" + std::to_string(k) +
                   (hop ? "_D" + std::to_string(D) : "") + "_" + std::to_string(s) + "-" +
                   std::to_string(e) + ".csv";
  FILE* f = std::fopen(fn.c_str(), "w");
  if (!f) {
    std::fprintf(stderr, "%s: cannot write %s\n", GST_PROGRAM, fn.c_str());
    return 1;
  }
  // column names exactly as each reference program writes them
  if (prog == "TrimCDP")
    std::fprintf(f, "task_ID,task,GPU1_nonHop_time,GPU_nonHop_cost,GPU_nonHop_memory,counts,process_num\n");
  else
    std::fprintf(f, "task_ID,task,%s_time,%s_cost,%s_memory,counts,process_num\n", tag.c_str(), tag.c_str(),
                 tag.c_str());
  int rc = 0;
  for (int i = 0; i < n; ++i) {
    std::string task;
    for (int64_t j = qs.ptr[s + i]; j < qs.ptr[s + i + 1]; ++j) task += std::to_string(qs.ids[j]) + " ";
    long long cost = res[i].cost;
    if (sts[i] != GST_OK) {
      std::fprintf(stderr, "%s: query %d failed: status %d\n", GST_PROGRAM, s + i, (int)sts[i]);
      rc = 1;
    }
    if (!res[i].feasible) cost = prog == "TrimCDP" ? 0 : GST_REF_INF;
    const int kk = (int)(qs.ptr[s + i + 1] - qs.ptr[s + i]);
    const long long width = (1ll << (kk < 31 ? kk : 30)) * (hop ? D + 1 : 1);
    std::fprintf(f, "%d,%s,%.8f,%lld,%lld,%lld,%lld\n", s + i, task.c_str(), res[i].stats.device_ms / 1e3, cost,
                 (long long)res[i].stats.touched * width, (long long)res[i].stats.touched,
                 (long long)res[i].stats.frontier);
    gst_result_free(&res[i]);
  }
  std::fprintf(f, "\n");
  std::fclose(f);
  gst_engine_destroy(eng);
  gst_csr_free(&g);
  gst_groups_free(&gr);
  gst_queries_free(&qs);
  return rc;
}
