// exec.cpp -- a plan executor over the C ABI: the part of Harmony's runtime that runs an
// RA plan's kernel sequence (Runtime.cpp:295-445: variables allocated at their first
// definition and freed after their last use, sizes read back where the next kernel is
// sized by them), with a JSON plan instead of the HIR protobuf.
//
// Plan:
//   { "variables": { "<name>": { "row_bytes": W }, ... },
//     "outputs": ["<name>", ...],
//     "ops": [ { "op": "<kind>", ... }, ... ] }
// Variables that no op defines are inputs: bound to caller memory (rfx_exec_bind) or
// loaded from a packed relation file (rfx_exec_load: the file is the relation's bytes,
// rows of row_bytes, as the reference's runtime reads a variable's file).  Op kinds:
//   sort        {rel, begin_bit, end_bit}                          in place
//   select      {in, out, widths, cmps}                            cmps: [{op, a, b, type}]
//   project     {in, out, widths, out_widths, map}
//   select_project {in, out, widths, cmps, out_widths, map}
//   join        {left, right, out, left_value_bits, right_value_bits, out_bytes}
//   reduce      {in, key_shift, value_shift, value_bits, keys, key_bytes, sums, counts}
//   set         {kind: union|difference|intersection, a, b, out}
//   unique      {rel}                                               in place
//   merge       {keys, values, out, value_bits}   out = key << value_bits | value (values
//               optional: then out = key); closes an aggregation as a relation
// A comparison operand is {"field": i} or {"const": c}.  Every device buffer comes from
// the stream-ordered allocator; the running total is held within the byte budget
// (RFX_ERR_CAPACITY otherwise) and its peak is reported.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "host_common.h"

namespace rfx {
namespace {

// ------------------------------------------------------------------ a small JSON reader
struct Json {
  enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
  bool b = false;
  double num = 0;
  long long inum = 0;
  bool is_int = false;
  std::string str;
  std::vector<Json> arr;
  std::vector<std::pair<std::string, Json>> obj;

  const Json* get(const std::string& k) const {
    for (const auto& kv : obj)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
};

struct JsonParser {
  const char* p;
  const char* end;
  std::string err;

  void ws() {
    while (p < end && (*p == ' ' || *p == '\n' || *p == '\t' || *p == '\r')) ++p;
  }
  bool fail(const char* m) {
    if (err.empty()) err = m;
    return false;
  }
  bool parse(Json& v) {
    ws();
    if (p >= end) return fail("unexpected end of plan");
    if (*p == '{') {
      v.kind = Json::OBJ;
      ++p;
      ws();
      if (p < end && *p == '}') return ++p, true;
      while (true) {
        ws();
        Json key;
        if (p >= end || *p != '"' || !parse(key)) return fail("expected a key");
        ws();
        if (p >= end || *p != ':') return fail("expected ':'");
        ++p;
        Json val;
        if (!parse(val)) return false;
        v.obj.emplace_back(key.str, std::move(val));
        ws();
        if (p < end && *p == ',') {
          ++p;
          continue;
        }
        if (p < end && *p == '}') return ++p, true;
        return fail("expected ',' or '}'");
      }
    }
    if (*p == '[') {
      v.kind = Json::ARR;
      ++p;
      ws();
      if (p < end && *p == ']') return ++p, true;
      while (true) {
        Json val;
        if (!parse(val)) return false;
        v.arr.push_back(std::move(val));
        ws();
        if (p < end && *p == ',') {
          ++p;
          continue;
        }
        if (p < end && *p == ']') return ++p, true;
        return fail("expected ',' or ']'");
      }
    }
    if (*p == '"') {
      v.kind = Json::STR;
      ++p;
      while (p < end && *p != '"') {
        if (*p == '\\' && p + 1 < end) ++p;
        v.str += *p++;
      }
      if (p >= end) return fail("unterminated string");
      return ++p, true;
    }
    if (!std::strncmp(p, "true", 4)) return v.kind = Json::BOOL, v.b = true, p += 4, true;
    if (!std::strncmp(p, "false", 5)) return v.kind = Json::BOOL, v.b = false, p += 5, true;
    if (!std::strncmp(p, "null", 4)) return v.kind = Json::NUL, p += 4, true;
    char* e = nullptr;
    const long long i = std::strtoll(p, &e, 10);
    if (e != p && (e >= end || (*e != '.' && *e != 'e' && *e != 'E'))) {
      v.kind = Json::NUM;
      v.inum = i;
      v.num = (double)i;
      v.is_int = true;
      p = e;
      return true;
    }
    const double d = std::strtod(p, &e);
    if (e == p) return fail("unexpected character in plan");
    v.kind = Json::NUM;
    v.num = d;
    v.inum = (long long)d;
    p = e;
    return true;
  }
};

// ------------------------------------------------------------------ plan
struct Var {
  std::string name;
  uint32_t row_bytes = 0;
  void* ptr = nullptr;      // device memory
  uint64_t bytes = 0;       // allocated bytes (0 for bound inputs)
  uint64_t rows = 0;        // logical rows
  bool input = false;       // defined by no op
  bool bound = false;       // caller memory
  bool output = false;
  bool in_arena = false;    // memory of the graph form's arena (never freed by itself)
  int last_use = -1;
  int def = -1;
};

struct Op {
  std::string kind;
  const Json* j;
  std::vector<std::string> reads, writes;
};

}  // namespace
}  // namespace rfx

struct rfx_exec {
  rfx::Json plan;
  std::map<std::string, rfx::Var> vars;
  std::vector<rfx::Op> ops;
  uint64_t budget = 0;
  uint64_t in_use = 0;
  uint64_t peak = 0;
  uint64_t launches = 0;   // operator calls
  std::string err;
  cudaStream_t stream = 0;
  // CUDA-graph form (rfx_exec_capture / rfx_exec_replay): an eager run records every
  // size read back and every allocation; the capture then takes its memory from one arena
  // in the same order and, where the eager run read a size back, copies the device count
  // into `observed` and uses the recorded size.  A replay is valid when every observed
  // size equals the recorded one.
  bool recording = false;
  bool capturing = false;
  std::vector<uint64_t> rec_sizes;
  std::vector<uint64_t> rec_allocs;
  size_t size_pos = 0;
  uint64_t arena_used = 0;
  void* arena = nullptr;
  uint64_t arena_bytes = 0;
  uint64_t* d_observed = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
};

namespace rfx {
namespace {

std::string jstr(const Json* j, const char* k) {
  const Json* v = j ? j->get(k) : nullptr;
  return v && v->kind == Json::STR ? v->str : std::string();
}
long long jint(const Json* j, const char* k, long long dflt = -1) {
  const Json* v = j ? j->get(k) : nullptr;
  return v && v->kind == Json::NUM ? v->inum : dflt;
}

rfx_status fail(rfx_exec* x, rfx_status st, const std::string& m) {
  x->err = m;
  return st;
}

// One allocation: from the stream-ordered allocator, or while capturing, the next block
// of the arena (allocations replay in the recorded order and are never freed inside
// the graph).
rfx_status raw_alloc(rfx_exec* x, void** p, uint64_t b) {
  if (x->capturing) {
    const uint64_t off = align_up(x->arena_used, 256);
    if (off + b > x->arena_bytes) return fail(x, RFX_ERR_CAPACITY, "capture: arena exhausted");
    *p = static_cast<uint8_t*>(x->arena) + off;
    x->arena_used = off + b;
    return RFX_OK;
  }
  if (x->recording) x->rec_allocs.push_back(b);
  RFX_CUDA_TRY(cudaMallocAsync(p, b, x->stream));
  return RFX_OK;
}

void raw_free(rfx_exec* x, void* p) {
  if (!x->capturing) cudaFreeAsync(p, x->stream);
}

rfx_status dev_alloc(rfx_exec* x, Var& v, uint64_t bytes) {
  const uint64_t b = bytes ? bytes : 16;
  if (x->budget && x->in_use + b > x->budget)
    return fail(x, RFX_ERR_CAPACITY, "memory budget exceeded allocating '" + v.name + "'");
  rfx_status st = raw_alloc(x, &v.ptr, b);
  if (st != RFX_OK) return st;
  v.in_arena = x->capturing;
  v.bytes = b;
  x->in_use += b;
  if (x->in_use > x->peak) x->peak = x->in_use;
  return RFX_OK;
}

void dev_free(rfx_exec* x, Var& v) {
  if (v.ptr && !v.bound) {
    if (!v.in_arena) raw_free(x, v.ptr);
    x->in_use -= v.bytes;
  }
  if (!v.bound) {
    v.ptr = nullptr;
    v.bytes = 0;
    v.in_arena = false;
  }
}

struct Scratch {  // temporary device memory counted against the budget
  rfx_exec* x;
  void* p = nullptr;
  uint64_t bytes = 0;
  ~Scratch() {
    if (p) {
      raw_free(x, p);
      x->in_use -= bytes;
    }
  }
  rfx_status alloc(uint64_t b) {
    bytes = b ? b : 16;
    if (x->budget && x->in_use + bytes > x->budget) {
      bytes = 0;
      return fail(x, RFX_ERR_CAPACITY, "memory budget exceeded allocating a workspace");
    }
    rfx_status st = raw_alloc(x, &p, bytes);
    if (st != RFX_OK) {
      p = nullptr;
      bytes = 0;
      return st;
    }
    x->in_use += bytes;
    if (x->in_use > x->peak) x->peak = x->in_use;
    return RFX_OK;
  }
};

rfx_status read_count(rfx_exec* x, const uint64_t* d, uint64_t* h) {
  if (x->capturing) {
    // the size the eager run read here; the replay's own count is kept for the check
    if (x->size_pos >= x->rec_sizes.size()) return fail(x, RFX_ERR_INVALID, "capture: plan diverged");
    RFX_CUDA_TRY(cudaMemcpyAsync(x->d_observed + x->size_pos, d, sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                                 x->stream));
    *h = x->rec_sizes[x->size_pos++];
    return RFX_OK;
  }
  RFX_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(uint64_t), cudaMemcpyDeviceToHost, x->stream));
  RFX_CUDA_TRY(cudaStreamSynchronize(x->stream));
  if (x->recording) x->rec_sizes.push_back(*h);
  return RFX_OK;
}

bool tuple_of(const Json* widths, rfx_tuple* t) {
  if (!widths || widths->kind != Json::ARR || widths->arr.empty() || widths->arr.size() > 16) return false;
  std::memset(t, 0, sizeof(*t));
  t->nfields = (uint32_t)widths->arr.size();
  for (size_t i = 0; i < widths->arr.size(); ++i) t->widths[i] = (uint32_t)widths->arr[i].inum;
  return true;
}

int cmp_code(const std::string& s) {
  static const char* names[] = {"", "eq", "ne", "slt", "lt", "sle", "le", "sgt", "gt", "sge", "ge"};
  for (int i = 1; i <= 10; ++i)
    if (s == names[i]) return i;
  return 0;
}
int type_code(const std::string& s) {
  static const char* names[] = {"", "i8", "i16", "i32", "i64", "i128", "i256", "i512"};
  for (int i = 1; i <= 7; ++i)
    if (s == names[i]) return i;
  return 0;
}

bool cmps_of(const Json* cmps, std::vector<rfx_cmp>& out) {
  if (!cmps) return true;
  if (cmps->kind != Json::ARR) return false;
  for (const Json& c : cmps->arr) {
    rfx_cmp r;
    std::memset(&r, 0, sizeof(r));
    r.op = (uint32_t)cmp_code(jstr(&c, "op"));
    r.value_type = (uint32_t)type_code(jstr(&c, "type"));
    if (!r.op || !r.value_type) return false;
    const Json* a = c.get("a");
    const Json* b = c.get("b");
    if (!a || !b) return false;
    if (a->get("field")) {
      r.a_kind = RFX_OPND_VARIABLE;
      r.a_field = (uint32_t)jint(a, "field");
    } else {
      r.a_kind = RFX_OPND_CONSTANT;
      r.a_const = (uint64_t)jint(a, "const", 0);
    }
    if (b->get("field")) {
      r.b_kind = RFX_OPND_VARIABLE;
      r.b_field = (uint32_t)jint(b, "field");
    } else {
      r.b_kind = RFX_OPND_CONSTANT;
      r.b_const = (uint64_t)jint(b, "const", 0);
    }
    out.push_back(r);
  }
  return true;
}

Var* var(rfx_exec* x, const std::string& n) {
  auto it = x->vars.find(n);
  return it == x->vars.end() ? nullptr : &it->second;
}

// ---- operators
rfx_status op_sort(rfx_exec* x, const Op& o) {
  Var* v = var(x, jstr(o.j, "rel"));
  const uint32_t w = v->row_bytes;
  const uint32_t b0 = (uint32_t)jint(o.j, "begin_bit", 0), b1 = (uint32_t)jint(o.j, "end_bit", w * 8);
  Scratch ws{x};
  const size_t need = rfx_sort_workspace(v->rows, w, 0, b0, b1);
  rfx_status st = ws.alloc(need);
  if (st != RFX_OK) return st;
  return rfx_sort_pairs(v->ptr, nullptr, v->rows, w, 0, b0, b1, 0, ws.p, need, x->stream);
}

rfx_status op_select_like(rfx_exec* x, const Op& o) {
  Var* in = var(x, jstr(o.j, "in"));
  Var* out = var(x, jstr(o.j, "out"));
  rfx_tuple t;
  if (!tuple_of(o.j->get("widths"), &t)) return fail(x, RFX_ERR_INVALID, o.kind + ": bad widths");
  std::vector<rfx_cmp> cm;
  if (!cmps_of(o.j->get("cmps"), cm)) return fail(x, RFX_ERR_INVALID, o.kind + ": bad cmps");
  rfx_tuple ot;
  std::vector<uint32_t> map;
  if (o.kind != "select") {
    if (!tuple_of(o.j->get("out_widths"), &ot)) return fail(x, RFX_ERR_INVALID, o.kind + ": bad out_widths");
    const Json* m = o.j->get("map");
    if (!m || m->kind != Json::ARR || m->arr.size() != ot.nfields) return fail(x, RFX_ERR_INVALID, o.kind + ": bad map");
    for (const Json& e : m->arr) map.push_back((uint32_t)e.inum);
  }
  rfx_status st = dev_alloc(x, *out, in->rows * (uint64_t)out->row_bytes);
  if (st != RFX_OK) return st;
  Scratch cnt{x}, ws{x};
  if ((st = cnt.alloc(sizeof(uint64_t))) != RFX_OK) return st;
  if (o.kind == "project") {
    st = rfx_project(out->ptr, in->ptr, in->rows, &t, &ot, map.data(), x->stream);
    out->rows = in->rows;
    return st;
  }
  const size_t need = rfx_select_workspace(in->rows, &t);
  if ((st = ws.alloc(need)) != RFX_OK) return st;
  if (o.kind == "select")
    st = rfx_select(out->ptr, (uint64_t*)cnt.p, in->ptr, in->rows, &t, cm.data(), (uint32_t)cm.size(), ws.p, need,
                    x->stream);
  else
    st = rfx_select_project(out->ptr, (uint64_t*)cnt.p, in->ptr, in->rows, &t, cm.data(), (uint32_t)cm.size(),
                            nullptr, 0, &ot, map.data(), ws.p, need, x->stream);
  if (st != RFX_OK) return st;
  return read_count(x, (const uint64_t*)cnt.p, &out->rows);
}

rfx_status op_join(rfx_exec* x, const Op& o) {
  Var* l = var(x, jstr(o.j, "left"));
  Var* r = var(x, jstr(o.j, "right"));
  Var* out = var(x, jstr(o.j, "out"));
  const uint32_t lv = (uint32_t)jint(o.j, "left_value_bits", 0), rv = (uint32_t)jint(o.j, "right_value_bits", 0);
  const uint32_t ob = out->row_bytes;
  Scratch ws{x}, cnt{x}, none{x};
  const size_t need = rfx_join_tuples_workspace(l->rows);
  rfx_status st = ws.alloc(need);
  if (st != RFX_OK || (st = cnt.alloc(sizeof(uint64_t))) != RFX_OK || (st = none.alloc(64)) != RFX_OK) return st;
  // count (capacity 0: nothing is written to `none`), read the size back, allocate
  // exactly, emit
  st = rfx_join_tuples(none.p, ob, 0, (uint64_t*)cnt.p, l->ptr, l->rows, l->row_bytes, lv, r->ptr, r->rows,
                       r->row_bytes, rv, ws.p, need, x->stream);
  if (st != RFX_OK) return st;
  uint64_t total = 0;
  if ((st = read_count(x, (const uint64_t*)cnt.p, &total)) != RFX_OK) return st;
  if ((st = dev_alloc(x, *out, total * ob)) != RFX_OK) return st;
  out->rows = total;
  return rfx_join_tuples_emit(out->ptr, ob, total, l->ptr, l->rows, l->row_bytes, r->ptr, r->rows, r->row_bytes, rv,
                              ws.p, need, x->stream);
}

rfx_status op_reduce(rfx_exec* x, const Op& o) {
  Var* in = var(x, jstr(o.j, "in"));
  Var* keys = var(x, jstr(o.j, "keys"));
  Var* sums = var(x, jstr(o.j, "sums"));
  Var* counts = var(x, jstr(o.j, "counts"));
  rfx_status st;
  // groups <= rows: every output sized by the input rows, the group count read back
  if ((st = dev_alloc(x, *keys, in->rows * (uint64_t)keys->row_bytes)) != RFX_OK) return st;
  if (sums && (st = dev_alloc(x, *sums, in->rows * 8ull)) != RFX_OK) return st;
  if (counts && (st = dev_alloc(x, *counts, in->rows * 4ull)) != RFX_OK) return st;
  Scratch ws{x}, g{x};
  const size_t need = rfx_reduce_by_key_workspace(in->rows);
  if ((st = ws.alloc(need)) != RFX_OK || (st = g.alloc(sizeof(uint64_t))) != RFX_OK) return st;
  st = rfx_reduce_tuples(in->ptr, in->rows, nullptr, in->row_bytes, (uint32_t)jint(o.j, "key_shift", 0),
                         (uint32_t)jint(o.j, "value_shift", 0), (uint32_t)jint(o.j, "value_bits", 64), keys->ptr,
                         keys->row_bytes, sums ? (int64_t*)sums->ptr : nullptr,
                         counts ? (uint32_t*)counts->ptr : nullptr, (uint64_t*)g.p, ws.p, need, x->stream);
  if (st != RFX_OK) return st;
  uint64_t groups = 0;
  if ((st = read_count(x, (const uint64_t*)g.p, &groups)) != RFX_OK) return st;
  keys->rows = groups;
  if (sums) sums->rows = groups;
  if (counts) counts->rows = groups;
  return RFX_OK;
}

rfx_status op_set(rfx_exec* x, const Op& o) {
  Var* a = var(x, jstr(o.j, "a"));
  Var* b = var(x, jstr(o.j, "b"));
  Var* out = var(x, jstr(o.j, "out"));
  const std::string k = jstr(o.j, "kind");
  const uint32_t op = k == "union" ? RFX_SET_UNION : k == "difference" ? RFX_SET_DIFFERENCE : RFX_SET_INTERSECTION;
  if (k != "union" && k != "difference" && k != "intersection") return fail(x, RFX_ERR_INVALID, "set: bad kind");
  if (a->row_bytes != b->row_bytes) return fail(x, RFX_ERR_INVALID, "set: element widths differ");
  const uint32_t e = a->row_bytes;
  rfx_status st = dev_alloc(x, *out, (a->rows + b->rows) * (uint64_t)e);
  if (st != RFX_OK) return st;
  Scratch ws{x}, cnt{x};
  const size_t need = rfx_set_op_workspace(op, a->rows, b->rows, e);
  if ((st = ws.alloc(need)) != RFX_OK || (st = cnt.alloc(sizeof(uint64_t))) != RFX_OK) return st;
  st = rfx_set_op(op, out->ptr, (uint64_t*)cnt.p, a->ptr, a->rows, b->ptr, b->rows, e, ws.p, need, x->stream);
  if (st != RFX_OK) return st;
  return read_count(x, (const uint64_t*)cnt.p, &out->rows);
}

rfx_status op_unique(rfx_exec* x, const Op& o) {
  Var* v = var(x, jstr(o.j, "rel"));
  Scratch ws{x}, cnt{x};
  const size_t need = rfx_unique_workspace(v->rows, v->row_bytes);
  rfx_status st = ws.alloc(need);
  if (st != RFX_OK || (st = cnt.alloc(sizeof(uint64_t))) != RFX_OK) return st;
  st = rfx_unique(v->ptr, v->rows, (uint64_t*)cnt.p, v->row_bytes, ws.p, need, x->stream);
  if (st != RFX_OK) return st;
  return read_count(x, (const uint64_t*)cnt.p, &v->rows);
}

rfx_status op_merge(rfx_exec* x, const Op& o) {
  Var* k = var(x, jstr(o.j, "keys"));
  Var* v = jstr(o.j, "values").empty() ? nullptr : var(x, jstr(o.j, "values"));
  Var* out = var(x, jstr(o.j, "out"));
  const uint32_t vb = v ? (uint32_t)jint(o.j, "value_bits", v->row_bytes * 8) : 0u;
  if (v && v->rows != k->rows) return fail(x, RFX_ERR_INVALID, "merge: column lengths differ");
  rfx_status st = dev_alloc(x, *out, k->rows * (uint64_t)out->row_bytes);
  if (st != RFX_OK) return st;
  out->rows = k->rows;
  return rfx_merge_columns(out->ptr, out->row_bytes, k->rows, nullptr, k->ptr, k->row_bytes, v ? v->ptr : nullptr,
                           v ? v->row_bytes : 4u, vb, x->stream);
}

void drop_graph(rfx_exec* x) {
  if (x->gexec) cudaGraphExecDestroy(x->gexec);
  if (x->graph) cudaGraphDestroy(x->graph);
  x->gexec = nullptr;
  x->graph = nullptr;
}

// reads / writes of an op (names), for liveness
bool op_operands(const Op& o, std::vector<std::string>& r, std::vector<std::string>& w) {
  const Json* j = o.j;
  if (o.kind == "sort" || o.kind == "unique") {
    r.push_back(jstr(j, "rel"));
    w.push_back(jstr(j, "rel"));
  } else if (o.kind == "select" || o.kind == "project" || o.kind == "select_project") {
    r.push_back(jstr(j, "in"));
    w.push_back(jstr(j, "out"));
  } else if (o.kind == "join") {
    r.push_back(jstr(j, "left"));
    r.push_back(jstr(j, "right"));
    w.push_back(jstr(j, "out"));
  } else if (o.kind == "reduce") {
    r.push_back(jstr(j, "in"));
    w.push_back(jstr(j, "keys"));
    if (!jstr(j, "sums").empty()) w.push_back(jstr(j, "sums"));
    if (!jstr(j, "counts").empty()) w.push_back(jstr(j, "counts"));
  } else if (o.kind == "set") {
    r.push_back(jstr(j, "a"));
    r.push_back(jstr(j, "b"));
    w.push_back(jstr(j, "out"));
  } else if (o.kind == "merge") {
    r.push_back(jstr(j, "keys"));
    if (!jstr(j, "values").empty()) r.push_back(jstr(j, "values"));
    w.push_back(jstr(j, "out"));
  } else {
    return false;
  }
  return true;
}

}  // namespace
}  // namespace rfx

using namespace rfx;

extern "C" rfx_status rfx_exec_create(rfx_exec** out, const char* plan_json, uint64_t budget_bytes, char* err,
                                      size_t err_cap) {
  if (!out || !plan_json) return RFX_ERR_INVALID;
  *out = nullptr;
  std::unique_ptr<rfx_exec> x(new rfx_exec());
  x->budget = budget_bytes;
  JsonParser ps{plan_json, plan_json + std::strlen(plan_json), ""};
  rfx_status st = RFX_OK;
  auto bad = [&](const std::string& m) {
    if (err && err_cap) {
      std::snprintf(err, err_cap, "%s", m.c_str());
    }
    st = RFX_ERR_INVALID;
  };
  if (!ps.parse(x->plan) || x->plan.kind != Json::OBJ) {
    bad("plan: " + (ps.err.empty() ? std::string("not an object") : ps.err));
    return st;
  }
  const Json* vars = x->plan.get("variables");
  const Json* ops = x->plan.get("ops");
  if (!vars || vars->kind != Json::OBJ || !ops || ops->kind != Json::ARR) {
    bad("plan: needs \"variables\" (object) and \"ops\" (array)");
    return st;
  }
  for (const auto& kv : vars->obj) {
    Var v;
    v.name = kv.first;
    v.row_bytes = (uint32_t)jint(&kv.second, "row_bytes", 0);
    if (v.row_bytes == 0) {
      bad("variable '" + kv.first + "': row_bytes missing");
      return st;
    }
    x->vars[v.name] = v;
  }
  for (size_t i = 0; i < ops->arr.size(); ++i) {
    Op o;
    o.j = &ops->arr[i];
    o.kind = jstr(o.j, "op");
    if (!op_operands(o, o.reads, o.writes)) {
      bad("op " + std::to_string(i) + ": unknown kind '" + o.kind + "'");
      return st;
    }
    for (const auto& n : o.reads) {
      Var* v = var(x.get(), n);
      if (!v) {
        bad("op " + std::to_string(i) + ": unknown variable '" + n + "'");
        return st;
      }
      if (v->def < 0) v->input = true;
      v->last_use = (int)i;
    }
    for (const auto& n : o.writes) {
      Var* v = var(x.get(), n);
      if (!v) {
        bad("op " + std::to_string(i) + ": unknown variable '" + n + "'");
        return st;
      }
      if (v->def < 0 && !v->input) v->def = (int)i;
      v->last_use = (int)i;
    }
    x->ops.push_back(o);
  }
  if (const Json* outs = x->plan.get("outputs")) {
    for (const Json& n : outs->arr) {
      Var* v = var(x.get(), n.str);
      if (!v) {
        bad("outputs: unknown variable '" + n.str + "'");
        return st;
      }
      v->output = true;
    }
  }
  *out = x.release();
  return RFX_OK;
}

extern "C" void rfx_exec_destroy(rfx_exec* x) {
  if (!x) return;
  for (auto& kv : x->vars) dev_free(x, kv.second);
  cudaStreamSynchronize(x->stream);
  drop_graph(x);
  if (x->arena) cudaFree(x->arena);
  if (x->d_observed) cudaFree(x->d_observed);
  delete x;
}

// Binds an input variable to caller device memory (`bytes` = the relation's bytes).
extern "C" rfx_status rfx_exec_bind(rfx_exec* x, const char* name, void* device_ptr, uint64_t bytes) {
  Var* v = x && name ? var(x, name) : nullptr;
  if (!v || !v->input || (bytes && !device_ptr) || bytes % v->row_bytes) return RFX_ERR_INVALID;
  v->ptr = device_ptr;
  v->rows = bytes / v->row_bytes;
  v->bound = true;
  return RFX_OK;
}

// Loads an input variable from a packed relation file (the relation's bytes, as the
// reference's runtime reads a variable's file, Runtime.cpp:191-206) into device memory
// owned by the executor.
extern "C" rfx_status rfx_exec_load(rfx_exec* x, const char* name, const char* path, void* stream) {
  Var* v = x && name && path ? var(x, name) : nullptr;
  if (!v || !v->input) return RFX_ERR_INVALID;
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) return fail(x, RFX_ERR_INVALID, std::string("cannot open ") + path);
  const uint64_t bytes = (uint64_t)f.tellg();
  if (bytes % v->row_bytes) return fail(x, RFX_ERR_INVALID, std::string(path) + ": size not a multiple of the row");
  f.seekg(0);
  std::vector<char> host(bytes);
  if (bytes && !f.read(host.data(), (std::streamsize)bytes)) return fail(x, RFX_ERR_INVALID, "read failed");
  x->stream = as_stream(stream);
  dev_free(x, *v);
  v->bound = false;
  rfx_status st = dev_alloc(x, *v, bytes);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaMemcpyAsync(v->ptr, host.data(), bytes, cudaMemcpyHostToDevice, x->stream));
  RFX_CUDA_TRY(cudaStreamSynchronize(x->stream));
  v->rows = bytes / v->row_bytes;
  return RFX_OK;
}

namespace rfx {
namespace {

// The op sequence: each defined variable is allocated at its op, every variable that is
// neither an input nor an output is freed after its last use.
rfx_status run_ops(rfx_exec* x) {
  for (auto& kv : x->vars) {
    Var& v = kv.second;
    if (v.input && !v.ptr && v.rows) return fail(x, RFX_ERR_INVALID, "input '" + v.name + "' not bound");
    if (v.input) continue;
    dev_free(x, v);   // a previous run's results
    v.rows = 0;
  }
  for (size_t i = 0; i < x->ops.size(); ++i) {
    const Op& o = x->ops[i];
    for (const auto& n : o.reads) {
      const Var* v = var(x, n);
      if (!v->ptr && v->rows) return fail(x, RFX_ERR_INVALID, "op " + std::to_string(i) + ": '" + n + "' has no data");
    }
    rfx_status st;
    if (o.kind == "sort") st = op_sort(x, o);
    else if (o.kind == "select" || o.kind == "project" || o.kind == "select_project") st = op_select_like(x, o);
    else if (o.kind == "join") st = op_join(x, o);
    else if (o.kind == "reduce") st = op_reduce(x, o);
    else if (o.kind == "set") st = op_set(x, o);
    else if (o.kind == "merge") st = op_merge(x, o);
    else st = op_unique(x, o);
    ++x->launches;
    if (st != RFX_OK) {
      if (x->err.empty()) x->err = "op " + std::to_string(i) + " (" + o.kind + ") failed";
      return st;
    }
    // liveness: free what no later op reads and nobody asked for
    for (auto& kv : x->vars) {
      Var& v = kv.second;
      if (!v.input && !v.output && v.last_use == (int)i) dev_free(x, v);
    }
  }
  return RFX_OK;
}

}  // namespace
}  // namespace rfx

// Runs the plan on `stream`.  Synchronises where an op's output size is needed (as the
// reference's GetSize / Resize kernels do).
extern "C" rfx_status rfx_exec_run(rfx_exec* x, void* stream) {
  if (!x) return RFX_ERR_INVALID;
  x->stream = as_stream(stream);
  rfx_status st = run_ops(x);
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(x->stream));
  return RFX_OK;
}

// Captures the plan as a CUDA graph on `stream` (not the legacy default stream): one eager
// run records the sizes it reads back and the allocations it makes; one arena of their
// total size is allocated (counted against the budget); the op sequence is then captured
// with its memory taken from the arena in the same order and the recorded sizes in place
// of the read-backs.  Inputs stay bound to the same memory; outputs live in the arena
// until the next capture or destroy.  Tuning (rfx_tune_set) must be off.
extern "C" rfx_status rfx_exec_capture(rfx_exec* x, void* stream) {
  if (!x) return RFX_ERR_INVALID;
  if (!stream) return fail(x, RFX_ERR_INVALID, "capture: needs a non-default stream");
  x->stream = as_stream(stream);
  drop_graph(x);
  x->rec_sizes.clear();
  x->rec_allocs.clear();
  x->recording = true;
  rfx_status st = run_ops(x);
  x->recording = false;
  if (st != RFX_OK) return st;
  RFX_CUDA_TRY(cudaStreamSynchronize(x->stream));
  for (auto& kv : x->vars)
    if (!kv.second.input) dev_free(x, kv.second);
  RFX_CUDA_TRY(cudaStreamSynchronize(x->stream));
  uint64_t need = 0;
  for (uint64_t b : x->rec_allocs) need = align_up(need, 256) + b;
  need = align_up(need, 256);
  if (x->arena) {
    x->in_use -= x->arena_bytes;
    cudaFree(x->arena);
    x->arena = nullptr;
    x->arena_bytes = 0;
  }
  if (x->d_observed) {
    cudaFree(x->d_observed);
    x->d_observed = nullptr;
  }
  if (x->budget && x->in_use + need > x->budget) return fail(x, RFX_ERR_CAPACITY, "capture: arena over the budget");
  RFX_CUDA_TRY(cudaMalloc(&x->arena, need ? need : 256));
  x->arena_bytes = need ? need : 256;
  x->in_use += x->arena_bytes;
  if (x->in_use > x->peak) x->peak = x->in_use;
  RFX_CUDA_TRY(cudaMalloc(&x->d_observed, (x->rec_sizes.size() + 1) * sizeof(uint64_t)));
  x->capturing = true;
  x->arena_used = 0;
  x->size_pos = 0;
  const uint64_t in_use0 = x->in_use;
  cudaError_t e = cudaStreamBeginCapture(x->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = run_ops(x);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(x->stream, &g);
    if (st == RFX_OK && e2 != cudaSuccess) st = cuda_fail(e2);
    if (st == RFX_OK) {
      x->graph = g;
      const cudaError_t e3 = cudaGraphInstantiate(&x->gexec, g, 0);
      if (e3 != cudaSuccess) {
        st = cuda_fail(e3);
        drop_graph(x);
      }
    } else if (g) {
      cudaGraphDestroy(g);
    }
  } else {
    st = cuda_fail(e);
  }
  x->capturing = false;
  x->in_use = in_use0;   // the arena holds everything; nothing else stays allocated
  return st;
}

// Replays the captured plan on `stream` and waits for it.  RFX_ERR_CAPACITY when an
// intermediate size differs from the captured one (the inputs' contents changed the
// plan's shape): the outputs are then invalid and the plan must run eagerly or be
// captured again.
extern "C" rfx_status rfx_exec_replay(rfx_exec* x, void* stream) {
  if (!x || !x->gexec) return RFX_ERR_INVALID;
  cudaStream_t s = as_stream(stream);
  RFX_CUDA_TRY(cudaGraphLaunch(x->gexec, s));
  std::vector<uint64_t> seen(x->rec_sizes.size());
  if (!seen.empty())
    RFX_CUDA_TRY(cudaMemcpyAsync(seen.data(), x->d_observed, seen.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost,
                                 s));
  RFX_CUDA_TRY(cudaStreamSynchronize(s));
  for (size_t i = 0; i < seen.size(); ++i)
    if (seen[i] != x->rec_sizes[i])
      return fail(x, RFX_ERR_CAPACITY, "replay: size " + std::to_string(i) + " is " + std::to_string(seen[i]) +
                                           ", captured " + std::to_string(x->rec_sizes[i]));
  ++x->launches;
  return RFX_OK;
}

// A variable's device pointer and logical size (rows x row_bytes) after a run.
extern "C" rfx_status rfx_exec_output(rfx_exec* x, const char* name, void** device_ptr, uint64_t* rows,
                                      uint32_t* row_bytes) {
  Var* v = x && name ? var(x, name) : nullptr;
  if (!v) return RFX_ERR_INVALID;
  if (device_ptr) *device_ptr = v->ptr;
  if (rows) *rows = v->rows;
  if (row_bytes) *row_bytes = v->row_bytes;
  return RFX_OK;
}

// Bytes held now and at the peak of the last runs, operator calls so far, and the last
// error message.
extern "C" rfx_status rfx_exec_stats(rfx_exec* x, uint64_t* in_use, uint64_t* peak, uint64_t* ops, char* err,
                                     size_t err_cap) {
  if (!x) return RFX_ERR_INVALID;
  if (in_use) *in_use = x->in_use;
  if (peak) *peak = x->peak;
  if (ops) *ops = x->launches;
  if (err && err_cap) std::snprintf(err, err_cap, "%s", x->err.c_str());
  return RFX_OK;
}

// Copies a variable's rows (after a run) into caller device memory of `cap_bytes`.
extern "C" rfx_status rfx_exec_copy_out(rfx_exec* x, const char* name, void* dst, uint64_t cap_bytes, void* stream) {
  Var* v = x && name ? var(x, name) : nullptr;
  if (!v) return RFX_ERR_INVALID;
  const uint64_t bytes = v->rows * v->row_bytes;
  if (bytes > cap_bytes || (bytes && (!dst || !v->ptr))) return RFX_ERR_CAPACITY;
  if (bytes) RFX_CUDA_TRY(cudaMemcpyAsync(dst, v->ptr, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)));
  return RFX_OK;
}
