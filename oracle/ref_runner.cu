// ref_runner.cu — drives the reference CUDA engine (harp-lab/gdlog-multinode,
// compiled unmodified from its own src/*.cu by oracle/Makefile) through its
// public API, for parity checks and as the GPU baseline.  TEST
// INFRASTRUCTURE ONLY: nothing in the product links or runs it.
//
//   ref_runner tc   <edges.tsv>
//   ref_runner sg   <edges.tsv>
//   ref_runner cspa <assign.tsv> <dereference.tsv>
//
// The programs are built exactly as the reference's own drivers build them
// (test/tc.cu:80-149, test/sg.cu:93-191, test/cspa.cu:100-379): same
// relations, load order, LIE membership and operators, with hooks that
// perform the same column moves.  The reference's own logging goes to
// stdout; this runner counts its "finish populating" lines (one per loop
// pass, src/lie.cu:199-200) to get each LIE's iteration count, and prints
// one result line on stderr:
//   REF {"program": ..., "sizes": {...}, "digests": {...},
//        "iterations": {...}, "seconds": S}
// The digest is the engine's order-sensitive digest of the sorted FULL
// tuples (gdlog-multinode_b200 gdl_relation_digest), computed here over
// the rows the reference's sorted FULL pointer array points at.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "exception.cuh"
#include "lie.cuh"

// -- hooks (column moves identical to the reference drivers') -------------
__device__ void h_inner1_outer1(tuple_type inner, tuple_type outer, tuple_type out) {
  out[0] = inner[1];
  out[1] = outer[1];
}
__device__ void h_outer1_inner1(tuple_type inner, tuple_type outer, tuple_type out) {
  out[0] = outer[1];
  out[1] = inner[1];
}
__device__ void c_swap(tuple_type src, tuple_type dst) {
  dst[0] = src[1];
  dst[1] = src[0];
}
__device__ void c_first_twice(tuple_type src, tuple_type dst) {
  dst[0] = src[0];
  dst[1] = src[0];
}
__device__ void c_second_twice(tuple_type src, tuple_type dst) {
  dst[0] = src[1];
  dst[1] = src[1];
}
__device__ bool p_not_equal(tuple_type t) { return t[0] != t[1]; }
// path_length's step: path(a, y, l + 1) from edge (x, a) reversed, path (x, y, l)
__device__ void h_path_step(tuple_type inner, tuple_type outer, tuple_type out) {
  out[0] = inner[1];
  out[1] = outer[1];
  out[2] = outer[2] + 1;
}
__device__ tuple_generator_hook d_path_step = h_path_step;

__device__ tuple_generator_hook d_inner1_outer1 = h_inner1_outer1;
__device__ tuple_generator_hook d_outer1_inner1 = h_outer1_inner1;
__device__ tuple_copy_hook d_swap = c_swap;
__device__ tuple_copy_hook d_first_twice = c_first_twice;
__device__ tuple_copy_hook d_second_twice = c_second_twice;
__device__ tuple_predicate d_not_equal = p_not_equal;

template <class T>
static T sym(const T &s) {
  T v;
  checkCuda(cudaMemcpyFromSymbol(&v, s, sizeof(T)));
  return v;
}

// -- input ----------------------------------------------------------------
static std::vector<column_type> read_tsv(const char *path) {
  std::vector<column_type> v;
  FILE *f = fopen(path, "r");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  unsigned long long a, b;
  while (fscanf(f, "%llu %llu", &a, &b) == 2) {
    v.push_back((column_type)a);
    v.push_back((column_type)b);
  }
  fclose(f);
  return v;
}
static std::vector<column_type> swapped(const std::vector<column_type> &v) {
  std::vector<column_type> r(v.size());
  for (size_t i = 0; i + 1 < v.size(); i += 2) {
    r[i] = v[i + 1];
    r[i + 1] = v[i];
  }
  return r;
}

// -- result digest ----------------------------------------------------------
__global__ void k_gather_rows(tuple_type *tuples, unsigned long long n, int arity,
                              unsigned long long *out) {
  for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    for (int c = 0; c < arity; c++) out[arity * i + c] = tuples[i][c];
}
static unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}
// Digest of FULL's tuples in the container's order (mix64 over the row
// index and every column); *sorted reports whether that order is strictly
// increasing.
static std::string digest_full(Relation *r, bool *sorted) {
  const int ar = r->arity;
  unsigned long long n = r->full->tuple_counts;
  std::vector<unsigned long long> h((size_t)ar * n);
  if (n) {
    unsigned long long *d;
    checkCuda(cudaMalloc(&d, (size_t)ar * n * sizeof(unsigned long long)));
    k_gather_rows<<<1024, 256>>>(r->full->tuples, n, ar, d);
    checkCuda(cudaGetLastError());
    checkCuda(cudaMemcpy(h.data(), d, (size_t)ar * n * sizeof(unsigned long long),
                         cudaMemcpyDeviceToHost));
    checkCuda(cudaFree(d));
  }
  unsigned long long acc = 0;
  *sorted = true;
  for (unsigned long long i = 0; i < n; i++) {
    if (i) {
      int c = 0;
      while (c < ar && h[ar * (i - 1) + c] == h[ar * i + c]) c++;
      if (c == ar || h[ar * (i - 1) + c] > h[ar * i + c]) *sorted = false;
    }
    unsigned long long x = mix64(i);
    for (int c = 0; c < ar; c++) x = mix64(x ^ h[ar * i + c]);
    acc += x;
  }
  char buf[32];
  snprintf(buf, sizeof buf, "0x%llx", mix64(acc ^ n));
  return buf;
}

// -- fixpoint with the reference's stdout captured ---------------------------
static double g_seconds = 0;
static unsigned long long run_lie(LIE &lie) {
  std::stringstream log;
  std::streambuf *old = std::cout.rdbuf(log.rdbuf());
  checkCuda(cudaDeviceSynchronize());
  auto t0 = std::chrono::steady_clock::now();
  lie.fixpoint_loop();
  checkCuda(cudaDeviceSynchronize());
  g_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::cout.rdbuf(old);
  unsigned long long passes = 0;
  std::string line;
  while (std::getline(log, line))
    if (line.find("finish populating") != std::string::npos) passes++;
  return passes;
}

static Relation *rel(const char *name, std::vector<column_type> *rows, bool index_flag = true,
                     bool tmp = false, int grid = 0, int block = 0) {
  Relation *r = new Relation();
  r->index_flag = index_flag;
  load_relation(r, name, 2, rows ? rows->data() : nullptr, rows ? rows->size() / 2 : 0, 1, 0, grid,
                block, tmp);
  return r;
}

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: ref_runner tc|sg|cspa <tsv> [<tsv>]\n");
    return 2;
  }
  int sms = 0;
  checkCuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  const int block = 512, grid = 32 * sms;  // launch shape of test/tc.cu:223-225
  std::string prog = argv[1];
  std::map<std::string, Relation *> out;
  std::map<std::string, unsigned long long> iters;
  std::streambuf *old = std::cout.rdbuf();
  std::stringstream sink;
  float detail[16] = {0};
  if (prog == "tc") {
    auto e = read_tsv(argv[2]);
    auto re = swapped(e);
    std::cout.rdbuf(sink.rdbuf());
    Relation *edge_2__2_1 = new Relation();
    Relation *path_2__1_2 = new Relation();
    path_2__1_2->index_flag = false;
    load_relation(path_2__1_2, "path_2__1_2", 2, e.data(), e.size() / 2, 1, 0, grid, block);
    load_relation(edge_2__2_1, "edge_2__2_1", 2, re.data(), re.size() / 2, 1, 0, grid, block);
    std::cout.rdbuf(old);
    LIE tc(grid, block);
    tc.reload_full_flag = false;
    tc.add_relations(edge_2__2_1, true);
    tc.add_relations(path_2__1_2, false);
    tc.add_ra(RelationalJoin(edge_2__2_1, FULL, path_2__1_2, DELTA, path_2__1_2,
                             sym(d_inner1_outer1), nullptr, LEFT, grid, block, detail));
    iters["tc"] = run_lie(tc);
    out["path"] = path_2__1_2;
  } else if (prog == "sg") {
    auto e = read_tsv(argv[2]);
    auto re = swapped(e);
    std::cout.rdbuf(sink.rdbuf());
    Relation *edge_2__1_2 = new Relation();
    Relation *edge_2__2_1 = rel("edge_2__2_1", &re, true, false, grid, block);
    Relation *sg = new Relation();
    sg->index_flag = false;
    load_relation(sg, "sg_2__2_1", 2, nullptr, 0, 1, 0, grid, block);
    load_relation(edge_2__1_2, "edge_2__1_2", 2, e.data(), e.size() / 2, 1, 0, grid, block);
    std::cout.rdbuf(old);
    (void)edge_2__2_1;
    LIE init(grid, block);
    init.add_relations(edge_2__1_2, true);
    init.add_relations(sg, false);
    init.add_ra(RelationalJoin(edge_2__1_2, FULL, edge_2__1_2, FULL, sg, sym(d_inner1_outer1),
                               sym(d_not_equal), LEFT, grid, block, detail));
    iters["init"] = run_lie(init);
    std::cout.rdbuf(sink.rdbuf());
    Relation *tmp = rel("tmp", nullptr, true, false, grid, block);
    tmp->index_flag = false;
    std::cout.rdbuf(old);
    LIE lie(grid, block);
    lie.add_relations(edge_2__1_2, true);
    lie.add_relations(sg, false);
    lie.add_tmp_relation(tmp);
    lie.add_ra(RelationalJoin(edge_2__1_2, FULL, sg, DELTA, tmp, sym(d_outer1_inner1), nullptr,
                              LEFT, grid, block, detail));
    lie.add_ra(RelationalJoin(edge_2__1_2, FULL, tmp, NEWT, sg, sym(d_outer1_inner1), nullptr,
                              LEFT, grid, block, detail));
    iters["sg"] = run_lie(lie);
    out["sg"] = sg;
  } else if (prog == "cspa" && argc >= 4) {
    auto as = read_tsv(argv[2]);
    auto de = read_tsv(argv[3]);
    auto ras = swapped(as), rde = swapped(de);
    std::cout.rdbuf(sink.rdbuf());
    Relation *assign_2__2_1 = rel("assign_2__2_1", &ras, true, false, grid, block);
    Relation *deref_2__1_2 = rel("dereference_2__1_2", &de, true, false, grid, block);
    Relation *deref_2__2_1 = rel("dereference_2__2_1", &rde, true, false, grid, block);
    Relation *vf12 = rel("value_flow_2__1_2", nullptr, true, false, grid, block);
    Relation *vf21 = rel("value_flow_2__2_1", nullptr, true, false, grid, block);
    Relation *ma12 = rel("memory_alias_2__1_2", nullptr, true, false, grid, block);
    Relation *ma21 = rel("memory_alias_2__2_1", nullptr, true, false, grid, block);
    std::cout.rdbuf(old);
    LIE init(grid, block);
    init.add_relations(vf12, false);
    init.add_relations(vf21, false);
    init.add_relations(ma12, false);
    init.add_relations(ma21, false);
    init.add_relations(assign_2__2_1, true);
    init.add_ra(RelationalCopy(assign_2__2_1, FULL, vf12, sym(d_first_twice), nullptr, grid, block));
    init.add_ra(RelationalCopy(assign_2__2_1, FULL, vf12, sym(d_second_twice), nullptr, grid, block));
    init.add_ra(RelationalCopy(assign_2__2_1, FULL, vf12, sym(d_swap), nullptr, grid, block));
    init.add_ra(RelationalCopy(assign_2__2_1, FULL, ma12, sym(d_first_twice), nullptr, grid, block));
    init.add_ra(RelationalCopy(assign_2__2_1, FULL, ma12, sym(d_second_twice), nullptr, grid, block));
    init.add_ra(RelationalCopy(vf12, DELTA, vf21, sym(d_swap), nullptr, grid, block));
    init.add_ra(RelationalCopy(ma12, DELTA, ma21, sym(d_swap), nullptr, grid, block));
    iters["init"] = run_lie(init);
    std::cout.rdbuf(sink.rdbuf());
    Relation *vff12 = rel("value_flow_forward_2__1_2", nullptr, true, false, grid, block);
    Relation *vff21 = rel("value_flow_forward_2__2_1", nullptr, true, false, grid, block);
    (void)vff12;
    (void)vff21;
    Relation *va12 = new Relation();
    va12->index_flag = false;
    load_relation(va12, "value_alias_2__1_2", 2, nullptr, 0, 1, 0, grid, block);
    Relation *tmp_def = new Relation();
    tmp_def->index_flag = false;
    load_relation(tmp_def, "tmp_rel_def", 2, nullptr, 0, 1, 0, grid, block);
    Relation *tmp_ma1 = new Relation();
    tmp_ma1->index_flag = false;
    load_relation(tmp_ma1, "tmp_rel_ma1", 2, nullptr, 0, 1, 0, grid, block, true);
    Relation *tmp_ma2 = new Relation();
    tmp_ma2->index_flag = false;
    load_relation(tmp_ma2, "tmp_rel_ma2", 2, nullptr, 0, 1, 0, grid, block, true);
    std::cout.rdbuf(old);
    auto i1o1 = sym(d_inner1_outer1), o1i1 = sym(d_outer1_inner1);
    LIE lie(grid, block);
    lie.add_relations(assign_2__2_1, true);
    lie.add_relations(deref_2__1_2, true);
    lie.add_relations(deref_2__2_1, true);
    lie.add_relations(vf12, false);
    lie.add_relations(vf21, false);
    lie.add_relations(ma12, false);
    lie.add_relations(ma21, false);
    lie.add_relations(va12, false);
    lie.add_tmp_relation(tmp_def);
    lie.add_tmp_relation(tmp_ma1);
    lie.add_tmp_relation(tmp_ma2);
    auto J = [&](Relation *in, RelationVersion iv, Relation *o, RelationVersion ov, Relation *res,
                 tuple_generator_hook h) {
      lie.add_ra(RelationalJoin(in, iv, o, ov, res, h, nullptr, LEFT, grid, block, detail));
    };
    J(vf12, FULL, vf21, DELTA, vf12, o1i1);
    J(vf21, FULL, vf12, DELTA, vf12, i1o1);
    J(vf12, FULL, vf12, DELTA, va12, i1o1);
    J(vf12, FULL, vf12, DELTA, va12, o1i1);
    J(assign_2__2_1, FULL, ma12, DELTA, vf12, i1o1);
    J(deref_2__1_2, FULL, va12, DELTA, tmp_def, o1i1);
    J(deref_2__1_2, FULL, tmp_def, NEWT, ma12, o1i1);
    J(ma12, FULL, vf12, DELTA, tmp_ma1, i1o1);
    J(vf12, FULL, ma12, DELTA, tmp_ma1, o1i1);
    J(vf12, FULL, tmp_ma1, NEWT, va12, o1i1);
    J(ma21, FULL, vf12, DELTA, tmp_ma2, i1o1);
    J(vf12, FULL, tmp_ma2, NEWT, va12, i1o1);
    lie.add_ra(RelationalACopy(vf12, vf21, sym(d_swap), nullptr, grid, block));
    lie.add_ra(RelationalACopy(ma12, ma21, sym(d_swap), nullptr, grid, block));
    iters["analysis"] = run_lie(lie);
    out["value_flow"] = vf12;
    out["memory_alias"] = ma12;
    out["value_alias"] = va12;
  } else if (prog == "plen") {
    // test/path_length.cu:59-140: path (x, y, 1) per edge, arity 3 with one
    // dependent column, joined with the reversed edges
    auto e = read_tsv(argv[2]);
    auto re = swapped(e);
    std::vector<column_type> p3;
    for (size_t i = 0; i + 1 < e.size(); i += 2) {
      p3.push_back(e[i]);
      p3.push_back(e[i + 1]);
      p3.push_back(1);
    }
    std::cout.rdbuf(sink.rdbuf());
    Relation *edge = rel("edge_2__2_1", &re, true, false, grid, block);
    Relation *path = new Relation();
    path->index_flag = false;
    load_relation(path, "path_3__1_2_3", 3, p3.data(), p3.size() / 3, 1, 1, grid, block);
    std::cout.rdbuf(old);
    LIE lie(grid, block);
    lie.add_relations(edge, true);
    lie.add_relations(path, false);
    lie.add_ra(RelationalJoin(edge, FULL, path, DELTA, path, sym(d_path_step), nullptr, LEFT, grid,
                              block, detail));
    iters["plen"] = run_lie(lie);
    out["path"] = path;
  } else {
    fprintf(stderr, "unknown program %s\n", prog.c_str());
    return 2;
  }
  std::string sizes, digests, its;
  bool all_sorted = true;
  for (auto &kv : out) {
    bool sorted = true;
    std::string d = digest_full(kv.second, &sorted);
    all_sorted &= sorted;
    sizes += (sizes.empty() ? "" : ", ") + ("\"" + kv.first + "\": ") +
             std::to_string(kv.second->full->tuple_counts);
    digests += (digests.empty() ? "" : ", ") + ("\"" + kv.first + "\": \"") + d + "\"";
  }
  for (auto &kv : iters)
    its += (its.empty() ? "" : ", ") + ("\"" + kv.first + "\": ") + std::to_string(kv.second);
  fprintf(stderr,
          "REF {\"program\": \"%s\", \"sizes\": {%s}, \"digests\": {%s}, \"iterations\": {%s}, "
          "\"sorted\": %s, \"seconds\": %.6f}\n",
          prog.c_str(), sizes.c_str(), digests.c_str(), its.c_str(), all_sorted ? "true" : "false",
          g_seconds);
  return 0;
}
