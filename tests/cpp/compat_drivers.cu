// compat_drivers.cu — the TC, SG and CSPA programs written against the
// drop-in C++ API (include/gdlog/), the way the reference's own drivers are
// written against its API (test/tc.cu, test/sg.cu, test/cspa.cu):
// __device__ hooks fetched with cudaMemcpyFromSymbol, Relation /
// load_relation / LIE / RelationalJoin / RelationalCopy / RelationalACopy.
//
//   compat_drivers tc   <edges.tsv>
//   compat_drivers sg   <edges.tsv>
//   compat_drivers cspa <assign.tsv> <dereference.tsv>
//   compat_drivers path_length <edges.tsv>   (arity 3, dependent column,
//                                             a hook that adds 1)
//   compat_drivers hook_max | hook_pred | hook_copy <edges.tsv>
//                      (hooks that are not column selections: run through
//                       their device function pointers)
//
// Prints one line: RESULT {"sizes": ..., "digests": ..., "iterations": ...}
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "gdlog/exception.cuh"
#include "gdlog/lie.cuh"
#include "gdlog/timer.cuh"

__device__ void join_i1_o1(tuple_type inner, tuple_type outer, tuple_type out) {
  out[0] = inner[1];
  out[1] = outer[1];
}
__device__ void join_o1_i1(tuple_type inner, tuple_type outer, tuple_type out) {
  out[1] = inner[1];
  out[0] = outer[1];
}
__device__ void copy_swap(tuple_type src, tuple_type dst) {
  dst[0] = src[1];
  dst[1] = src[0];
}
__device__ void copy_c0c0(tuple_type src, tuple_type dst) {
  dst[0] = src[0];
  dst[1] = src[0];
}
__device__ void copy_c1c1(tuple_type src, tuple_type dst) {
  dst[0] = src[1];
  dst[1] = src[1];
}
__device__ bool not_equal(tuple_type t) { return t[0] != t[1]; }
// path(a, y, l + 1) from edge (x, a) reversed and path (x, y, l)
__device__ void path_step(tuple_type inner, tuple_type outer, tuple_type out) {
  out[0] = inner[1];
  out[1] = outer[1];
  out[2] = outer[2] + 1;
}
__device__ tuple_generator_hook path_step_d = path_step;

// Hooks that are not column selections: the engine runs them through
// their function pointers, as the reference does.
__device__ void join_max(tuple_type inner, tuple_type outer, tuple_type out) {
  out[0] = inner[1] > outer[1] ? inner[1] : outer[1];
  out[1] = outer[1];
}
__device__ bool ne_and_below(tuple_type t) { return t[0] != t[1] && t[0] < 100; }
__device__ void copy_xor(tuple_type src, tuple_type dst) {
  dst[0] = src[1];
  dst[1] = src[0] ^ 1;
}
__device__ void copy_swap_xor(tuple_type src, tuple_type dst) {
  dst[0] = src[1] ^ 1;
  dst[1] = src[0];
}
__device__ tuple_generator_hook join_max_d = join_max;
__device__ tuple_predicate ne_and_below_d = ne_and_below;
__device__ tuple_copy_hook copy_xor_d = copy_xor;
__device__ tuple_copy_hook copy_swap_xor_d = copy_swap_xor;

__device__ tuple_generator_hook join_i1_o1_d = join_i1_o1;
__device__ tuple_generator_hook join_o1_i1_d = join_o1_i1;
__device__ tuple_copy_hook copy_swap_d = copy_swap;
__device__ tuple_copy_hook copy_c0c0_d = copy_c0c0;
__device__ tuple_copy_hook copy_c1c1_d = copy_c1c1;
__device__ tuple_predicate not_equal_d = not_equal;

template <class T>
static T fetch(const T &sym) {
  T h;
  checkCuda(cudaMemcpyFromSymbol(&h, sym, sizeof(T)));
  return h;
}

static std::vector<column_type> read_tsv(const char *path) {
  std::vector<column_type> v;
  FILE *f = fopen(path, "r");
  if (!f) {
    fprintf(stderr, "cannot open %s\n", path);
    exit(2);
  }
  unsigned long a, b;
  while (fscanf(f, "%lu %lu", &a, &b) == 2) {
    v.push_back(a);
    v.push_back(b);
  }
  fclose(f);
  return v;
}

static std::vector<column_type> swap_cols(const std::vector<column_type> &v) {
  std::vector<column_type> r(v.size());
  for (size_t i = 0; i + 1 < v.size(); i += 2) {
    r[i] = v[i + 1];
    r[i + 1] = v[i];
  }
  return r;
}

static void load(Relation *r, const char *name, std::vector<column_type> *rows, bool tmp = false) {
  load_relation(r, name, 2, rows ? rows->data() : nullptr, rows ? rows->size() / 2 : 0, 1, 0, 0,
                0, tmp);
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  const std::string prog = argv[1];
  const int grid = 0, block = 512;
  float detail[10] = {0};
  std::map<std::string, Relation *> out;
  std::map<std::string, unsigned long long> iters;
  if (prog == "tc") {
    auto e = read_tsv(argv[2]);
    auto re = swap_cols(e);
    Relation *edge = new Relation();
    Relation *path = new Relation();
    path->index_flag = false;
    load(path, "path_2__1_2", &e);
    load(edge, "edge_2__2_1", &re);
    LIE tc(grid, block);
    tc.reload_full_flag = false;
    tc.add_relations(edge, true);
    tc.add_relations(path, false);
    tc.add_ra(RelationalJoin(edge, FULL, path, DELTA, path, fetch(join_i1_o1_d), nullptr, LEFT,
                             grid, block, detail));
    tc.fixpoint_loop();
    iters["tc"] = tc.iteration_counter;
    out["path"] = path;
  } else if (prog == "hook_max") {
    // path(max(x, z), z) :- edge(x, y), path(y, z): a generator that
    // compares columns.
    auto e = read_tsv(argv[2]);
    auto re = swap_cols(e);
    Relation *edge = new Relation();
    Relation *path = new Relation();
    path->index_flag = false;
    load(path, "path_2__1_2", &e);
    load(edge, "edge_2__2_1", &re);
    LIE lie(grid, block);
    lie.add_relations(edge, true);
    lie.add_relations(path, false);
    lie.add_ra(RelationalJoin(edge, FULL, path, DELTA, path, fetch(join_max_d), nullptr, LEFT,
                              grid, block, detail));
    lie.fixpoint_loop();
    iters["lie"] = lie.iteration_counter;
    out["path"] = path;
  } else if (prog == "hook_pred") {
    // same generation's first rule with the predicate t0 != t1 && t0 < 100,
    // then the recursive rules as in test/sg.cu
    auto e = read_tsv(argv[2]);
    Relation *edge12 = new Relation(), *sg = new Relation(), *tmp = new Relation();
    sg->index_flag = false;
    load(edge12, "edge_2__1_2", &e);
    load(sg, "sg_2__2_1", nullptr);
    LIE init(grid, block);
    init.add_relations(edge12, true);
    init.add_relations(sg, false);
    init.add_ra(RelationalJoin(edge12, FULL, edge12, FULL, sg, fetch(join_i1_o1_d),
                               fetch(ne_and_below_d), LEFT, grid, block, detail));
    init.fixpoint_loop();
    load(tmp, "tmp", nullptr);
    tmp->index_flag = false;
    LIE lie(grid, block);
    lie.add_relations(edge12, true);
    lie.add_relations(sg, false);
    lie.add_tmp_relation(tmp);
    lie.add_ra(RelationalJoin(edge12, FULL, sg, DELTA, tmp, fetch(join_o1_i1_d), nullptr, LEFT,
                              grid, block, detail));
    lie.add_ra(RelationalJoin(edge12, FULL, tmp, NEWT, sg, fetch(join_o1_i1_d),
                              fetch(ne_and_below_d), LEFT, grid, block, detail));
    lie.fixpoint_loop();
    iters["init"] = init.iteration_counter;
    iters["lie"] = lie.iteration_counter;
    out["sg"] = sg;
  } else if (prog == "hook_copy") {
    // r seeded by a copy hook that flips a bit, closed under the edges;
    // m the ACopy of r's NEWT through another such hook; d a copy of r's
    // DELTA through the first.
    auto e = read_tsv(argv[2]);
    auto re = swap_cols(e);
    Relation *edge = new Relation(), *r = new Relation(), *m = new Relation(),
             *d = new Relation();
    load(edge, "edge_2__2_1", &re);
    load(r, "r", nullptr);
    load(m, "m", nullptr);
    load(d, "d", nullptr);
    LIE lie(grid, block);
    lie.add_relations(edge, true);
    lie.add_relations(r, false);
    lie.add_relations(m, false);
    lie.add_relations(d, false);
    lie.add_ra(RelationalCopy(edge, FULL, r, fetch(copy_xor_d), nullptr, grid, block));
    lie.add_ra(RelationalJoin(edge, FULL, r, DELTA, r, fetch(join_i1_o1_d), nullptr, LEFT, grid,
                              block, detail));
    lie.add_ra(RelationalCopy(r, DELTA, d, fetch(copy_xor_d), nullptr, grid, block));
    lie.add_ra(RelationalACopy(r, m, fetch(copy_swap_xor_d), nullptr, grid, block));
    lie.fixpoint_loop();
    iters["lie"] = lie.iteration_counter;
    out["r"] = r;
    out["m"] = m;
    out["d"] = d;
  } else if (prog == "sg") {
    auto e = read_tsv(argv[2]);
    auto re = swap_cols(e);
    Relation *edge12 = new Relation(), *edge21 = new Relation(), *sg = new Relation();
    load(edge21, "edge_2__2_1", &re);
    sg->index_flag = false;
    load(sg, "sg_2__2_1", nullptr);
    load(edge12, "edge_2__1_2", &e);
    LIE init(grid, block);
    init.add_relations(edge12, true);
    init.add_relations(sg, false);
    init.add_ra(RelationalJoin(edge12, FULL, edge12, FULL, sg, fetch(join_i1_o1_d),
                               fetch(not_equal_d), LEFT, grid, block, detail));
    init.fixpoint_loop();
    Relation *tmp = new Relation();
    load(tmp, "tmp", nullptr);
    tmp->index_flag = false;
    LIE lie(grid, block);
    lie.add_relations(edge12, true);
    lie.add_relations(sg, false);
    lie.add_tmp_relation(tmp);
    lie.add_ra(RelationalJoin(edge12, FULL, sg, DELTA, tmp, fetch(join_o1_i1_d), nullptr, LEFT,
                              grid, block, detail));
    lie.add_ra(RelationalJoin(edge12, FULL, tmp, NEWT, sg, fetch(join_o1_i1_d), nullptr, LEFT,
                              grid, block, detail));
    lie.fixpoint_loop();
    iters["init"] = init.iteration_counter;
    iters["sg"] = lie.iteration_counter;
    out["sg"] = sg;
  } else if (prog == "path_length") {
    auto e = read_tsv(argv[2]);
    auto re = swap_cols(e);
    std::vector<column_type> p3;
    for (size_t i = 0; i + 1 < e.size(); i += 2) {
      p3.push_back(e[i]);
      p3.push_back(e[i + 1]);
      p3.push_back(1);
    }
    Relation *edge = new Relation(), *path = new Relation();
    path->index_flag = false;
    load_relation(path, "path_3__1_2_3", 3, p3.data(), p3.size() / 3, 1, 1, 0, 0);
    load(edge, "edge_2__2_1", &re);
    LIE plen(grid, block);
    plen.add_relations(edge, true);
    plen.add_relations(path, false);
    plen.add_ra(RelationalJoin(edge, FULL, path, DELTA, path, fetch(path_step_d), nullptr, LEFT,
                               grid, block, detail));
    plen.fixpoint_loop();
    iters["plen"] = plen.iteration_counter;
    out["path"] = path;
  } else if (prog == "cspa" && argc >= 4) {
    auto as = read_tsv(argv[2]), de = read_tsv(argv[3]);
    auto ras = swap_cols(as), rde = swap_cols(de);
    Relation *assign21 = new Relation(), *deref12 = new Relation(), *deref21 = new Relation();
    load(assign21, "assign_2__2_1", &ras);
    load(deref12, "dereference_2__1_2", &de);
    load(deref21, "dereference_2__2_1", &rde);
    Relation *vf12 = new Relation(), *vf21 = new Relation(), *ma12 = new Relation(),
             *ma21 = new Relation();
    load(vf12, "value_flow_2__1_2", nullptr);
    load(vf21, "value_flow_2__2_1", nullptr);
    load(ma12, "memory_alias_2__1_2", nullptr);
    load(ma21, "memory_alias_2__2_1", nullptr);
    LIE init(grid, block);
    for (Relation *r : {vf12, vf21, ma12, ma21}) init.add_relations(r, false);
    init.add_relations(assign21, true);
    auto c00 = fetch(copy_c0c0_d), c11 = fetch(copy_c1c1_d), sw = fetch(copy_swap_d);
    init.add_ra(RelationalCopy(assign21, FULL, vf12, c00, nullptr, grid, block));
    init.add_ra(RelationalCopy(assign21, FULL, vf12, c11, nullptr, grid, block));
    init.add_ra(RelationalCopy(assign21, FULL, vf12, sw, nullptr, grid, block));
    init.add_ra(RelationalCopy(assign21, FULL, ma12, c00, nullptr, grid, block));
    init.add_ra(RelationalCopy(assign21, FULL, ma12, c11, nullptr, grid, block));
    init.add_ra(RelationalCopy(vf12, DELTA, vf21, sw, nullptr, grid, block));
    init.add_ra(RelationalCopy(ma12, DELTA, ma21, sw, nullptr, grid, block));
    init.fixpoint_loop();
    Relation *va12 = new Relation(), *tdef = new Relation(), *tma1 = new Relation(),
             *tma2 = new Relation();
    va12->index_flag = tdef->index_flag = tma1->index_flag = tma2->index_flag = false;
    load(va12, "value_alias_2__1_2", nullptr);
    load(tdef, "tmp_rel_def", nullptr);
    load(tma1, "tmp_rel_ma1", nullptr, true);
    load(tma2, "tmp_rel_ma2", nullptr, true);
    auto i1o1 = fetch(join_i1_o1_d), o1i1 = fetch(join_o1_i1_d);
    LIE lie(grid, block);
    for (Relation *r : {assign21, deref12, deref21}) lie.add_relations(r, true);
    for (Relation *r : {vf12, vf21, ma12, ma21, va12}) lie.add_relations(r, false);
    for (Relation *r : {tdef, tma1, tma2}) lie.add_tmp_relation(r);
    auto J = [&](Relation *in, RelationVersion iv, Relation *o, RelationVersion ov, Relation *res,
                 tuple_generator_hook h) {
      lie.add_ra(RelationalJoin(in, iv, o, ov, res, h, nullptr, LEFT, grid, block, detail));
    };
    J(vf12, FULL, vf21, DELTA, vf12, o1i1);
    J(vf21, FULL, vf12, DELTA, vf12, i1o1);
    J(vf12, FULL, vf12, DELTA, va12, i1o1);
    J(vf12, FULL, vf12, DELTA, va12, o1i1);
    J(assign21, FULL, ma12, DELTA, vf12, i1o1);
    J(deref12, FULL, va12, DELTA, tdef, o1i1);
    J(deref12, FULL, tdef, NEWT, ma12, o1i1);
    J(ma12, FULL, vf12, DELTA, tma1, i1o1);
    J(vf12, FULL, ma12, DELTA, tma1, o1i1);
    J(vf12, FULL, tma1, NEWT, va12, o1i1);
    J(ma21, FULL, vf12, DELTA, tma2, i1o1);
    J(vf12, FULL, tma2, NEWT, va12, i1o1);
    lie.add_ra(RelationalACopy(vf12, vf21, sw, nullptr, grid, block));
    lie.add_ra(RelationalACopy(ma12, ma21, sw, nullptr, grid, block));
    lie.fixpoint_loop();
    iters["init"] = init.iteration_counter;
    iters["analysis"] = lie.iteration_counter;
    out["value_flow"] = vf12;
    out["memory_alias"] = ma12;
    out["value_alias"] = va12;
  } else {
    return 2;
  }
  std::string s = "RESULT {\"sizes\": {", d = "\"digests\": {", it = "\"iterations\": {";
  bool first = true;
  for (auto &kv : out) {
    char buf[64];
    snprintf(buf, sizeof buf, "\"0x%llx\"", (unsigned long long)kv.second->digest());
    s += (first ? "\"" : ", \"") + kv.first + "\": " + std::to_string(kv.second->full->tuple_counts);
    d += (first ? "\"" : ", \"") + kv.first + "\": " + buf;
    first = false;
  }
  first = true;
  for (auto &kv : iters) {
    it += (first ? "\"" : ", \"") + kv.first + "\": " + std::to_string(kv.second);
    first = false;
  }
  printf("%s}, %s}, %s}}\n", s.c_str(), d.c_str(), it.c_str());
  return 0;
}
