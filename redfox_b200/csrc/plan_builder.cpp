// plan_builder.cpp -- lowers relational-algebra operators to an executor plan: the job of
// the reference's RelationalAlgebraCompiler (addJoin :4466-5227, addAgg :7852-8643, and the
// select / project / set-operation builders) without protobuf and without compiling kernels
// at run time.  The caller declares relations (field widths, field 0 most significant, and
// how many leading fields they are sorted on) and adds operators; rfx_plan_json returns the
// plan that rfx_exec_create runs.
//
// Lowering, per operator, following the reference's sequences and their sortedness
// tracking (VariableMap's isSorted / sorted_fields):
//   select(d, s, cmps)        select; d keeps s's order.  A select read only by one
//                             project becomes one select_project (a single pass).
//   project(d, s, fields)     project (the reference's reordering / projection).
//   join(d, a, b, k)          keys are the first k fields of both (the RA convention);
//                             an input not sorted on them is sorted in place on its key
//                             bits (addSortPair / addSortKey); then one fused join, whose
//                             rows are key, a's other fields, b's other fields -- the
//                             reference's split + find_bounds + join + gather.
//   agg(d, s, domains, COUNT | TOTAL field)
//                             when the domains are s's leading fields, reduce reads the key
//                             and the summed field straight from s's rows (no projection,
//                             no split); otherwise s is projected to (domains, field) first.
//                             Unsorted input is sorted on the key bits; a COUNT over the
//                             same input and domains as an earlier TOTAL shares its reduce.
//                             The key and value columns are merged back into d = (domains,
//                             value): TOTAL values are exact 64-bit sums, COUNT 32-bit.
//   union / difference / intersection(d, a, b), unique(s)
//                             inputs sorted on all fields first (sorted in place if not).
// Sorting an input in place changes that relation's row order for the rest of the plan, as
// the reference's in-place sorts do; the builder records the new order and sorts once.
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "rfx/rfx.h"

namespace {

struct Rel {
  std::vector<uint32_t> widths;
  uint32_t sorted = 0;   // leading fields the rows are sorted on
  uint32_t version = 0;  // bumped when the rows are reordered in place
  bool input = false;
};

// One op of the executor plan: ordered (key, JSON value) pairs.
struct POp {
  std::vector<std::pair<std::string, std::string>> kv;
  const std::string* get(const std::string& k) const {
    for (const auto& p : kv)
      if (p.first == k) return &p.second;
    return nullptr;
  }
  void set(const std::string& k, const std::string& v) {
    for (auto& p : kv)
      if (p.first == k) {
        p.second = v;
        return;
      }
    kv.emplace_back(k, v);
  }
};

struct AggShare {
  size_t reduce_op;   // index of the reduce op
  std::string src;
  uint32_t version;
  std::vector<uint32_t> domains;
  int total_field;    // -1: none
  std::string keys, sums, counts;
};

uint32_t total_bits(const std::vector<uint32_t>& w) {
  uint32_t t = 0;
  for (uint32_t x : w) t += x;
  return t;
}

uint32_t container(uint32_t bits) {
  for (uint32_t c : {8u, 16u, 32u, 64u, 128u, 256u, 512u})
    if (bits <= c) return c / 8;
  return 0;
}

std::string q(const std::string& s) { return "\"" + s + "\""; }

std::string arr(const std::vector<uint32_t>& v) {
  std::string s = "[";
  for (size_t i = 0; i < v.size(); ++i) s += (i ? ", " : "") + std::to_string(v[i]);
  return s + "]";
}

const char* cmp_name(uint32_t op) {
  static const char* n[] = {"", "eq", "ne", "slt", "lt", "sle", "le", "sgt", "gt", "sge", "ge"};
  return op >= 1 && op <= 10 ? n[op] : nullptr;
}

const char* type_name(uint32_t t) {
  static const char* n[] = {"", "i8", "i16", "i32", "i64", "i128", "i256", "i512"};
  return t >= 1 && t <= 7 ? n[t] : nullptr;
}

}  // namespace

struct rfx_plan {
  std::map<std::string, Rel> rels;
  std::map<std::string, uint32_t> vars;  // executor variables: name -> row bytes
  std::vector<POp> ops;
  std::vector<std::string> outputs;
  std::vector<AggShare> shares;
  std::string err;

  rfx_status fail(rfx_status st, const std::string& m) {
    err = m;
    return st;
  }
  Rel* rel(const char* name) {
    if (!name) return nullptr;
    auto it = rels.find(name);
    return it == rels.end() ? nullptr : &it->second;
  }
  bool fresh(const char* name) const { return name && *name && !rels.count(name) && !vars.count(name); }
  void define(const std::string& name, const Rel& r) {
    rels[name] = r;
    vars[name] = container(total_bits(r.widths));
  }
  // Sort `name` in place on fields [0, k) (the bits above its remaining fields).
  void sort_on(const std::string& name, Rel& r, uint32_t k) {
    uint32_t low = 0;
    for (size_t i = k; i < r.widths.size(); ++i) low += r.widths[i];
    POp o;
    o.kv = {{"op", q("sort")}, {"rel", q(name)}, {"begin_bit", std::to_string(low)},
            {"end_bit", std::to_string(total_bits(r.widths))}};
    ops.push_back(o);
    r.sorted = k;
    ++r.version;
  }
};

extern "C" {

rfx_status rfx_plan_create(rfx_plan** out) {
  if (!out) return RFX_ERR_INVALID;
  *out = new rfx_plan();
  return RFX_OK;
}

void rfx_plan_destroy(rfx_plan* p) { delete p; }

const char* rfx_plan_error(const rfx_plan* p) { return p ? p->err.c_str() : ""; }

rfx_status rfx_plan_relation(rfx_plan* p, const char* name, const uint32_t* widths, uint32_t nfields,
                             uint32_t sorted_fields) {
  if (!p || !widths || nfields == 0 || nfields > 16) return RFX_ERR_INVALID;
  if (!p->fresh(name)) return p->fail(RFX_ERR_INVALID, std::string("relation name in use or empty: ") + (name ? name : ""));
  Rel r;
  r.widths.assign(widths, widths + nfields);
  for (uint32_t w : r.widths)
    if (w == 0 || w > 64) return p->fail(RFX_ERR_INVALID, "field widths must be 1..64 bits");
  if (container(total_bits(r.widths)) == 0) return p->fail(RFX_ERR_UNSUPPORTED, "tuple wider than 512 bits");
  r.sorted = sorted_fields < nfields ? sorted_fields : nfields;
  r.input = true;
  p->define(name, r);
  return RFX_OK;
}

rfx_status rfx_plan_select(rfx_plan* p, const char* dest, const char* src, const rfx_cmp* cmps, uint32_t ncmp) {
  if (!p || (ncmp && !cmps)) return RFX_ERR_INVALID;
  Rel* s = p->rel(src);
  if (!s) return p->fail(RFX_ERR_INVALID, std::string("select: unknown relation ") + (src ? src : ""));
  if (!p->fresh(dest)) return p->fail(RFX_ERR_INVALID, "select: destination name in use or empty");
  std::string cj = "[";
  for (uint32_t i = 0; i < ncmp; ++i) {
    const rfx_cmp& c = cmps[i];
    if (!cmp_name(c.op) || !type_name(c.value_type)) return p->fail(RFX_ERR_INVALID, "select: bad comparison code");
    auto opnd = [&](uint32_t kind, uint32_t field, uint64_t k, std::string* o) {
      if (kind == RFX_OPND_VARIABLE) {
        if (field >= s->widths.size()) return false;
        *o = "{\"field\": " + std::to_string(field) + "}";
      } else {
        *o = "{\"const\": " + std::to_string(k) + "}";
      }
      return true;
    };
    std::string a, b;
    if (!opnd(c.a_kind, c.a_field, c.a_const, &a) || !opnd(c.b_kind, c.b_field, c.b_const, &b))
      return p->fail(RFX_ERR_INVALID, "select: field index out of range");
    cj += std::string(i ? ", " : "") + "{\"op\": " + q(cmp_name(c.op)) + ", \"a\": " + a + ", \"b\": " + b +
          ", \"type\": " + q(type_name(c.value_type)) + "}";
  }
  cj += "]";
  POp o;
  o.kv = {{"op", q("select")}, {"in", q(src)}, {"out", q(dest)}, {"widths", arr(s->widths)}, {"cmps", cj}};
  p->ops.push_back(o);
  Rel d = *s;
  d.input = false;
  d.version = 0;
  p->define(dest, d);
  return RFX_OK;
}

rfx_status rfx_plan_project(rfx_plan* p, const char* dest, const char* src, const uint32_t* fields, uint32_t nfields) {
  if (!p || !fields || nfields == 0 || nfields > 16) return RFX_ERR_INVALID;
  Rel* s = p->rel(src);
  if (!s) return p->fail(RFX_ERR_INVALID, std::string("project: unknown relation ") + (src ? src : ""));
  if (!p->fresh(dest)) return p->fail(RFX_ERR_INVALID, "project: destination name in use or empty");
  Rel d;
  for (uint32_t i = 0; i < nfields; ++i) {
    if (fields[i] >= s->widths.size()) return p->fail(RFX_ERR_INVALID, "project: field index out of range");
    d.widths.push_back(s->widths[fields[i]]);
  }
  while (d.sorted < nfields && d.sorted < s->sorted && fields[d.sorted] == d.sorted) ++d.sorted;
  POp o;
  o.kv = {{"op", q("project")},
          {"in", q(src)},
          {"out", q(dest)},
          {"widths", arr(s->widths)},
          {"out_widths", arr(d.widths)},
          {"map", arr(std::vector<uint32_t>(fields, fields + nfields))}};
  p->ops.push_back(o);
  p->define(dest, d);
  return RFX_OK;
}

rfx_status rfx_plan_join(rfx_plan* p, const char* dest, const char* a, const char* b, uint32_t keycount) {
  if (!p) return RFX_ERR_INVALID;
  Rel* l = p->rel(a);
  Rel* r = p->rel(b);
  if (!l || !r) return p->fail(RFX_ERR_INVALID, "join: unknown relation");
  if (!p->fresh(dest)) return p->fail(RFX_ERR_INVALID, "join: destination name in use or empty");
  if (keycount == 0 || keycount > l->widths.size() || keycount > r->widths.size())
    return p->fail(RFX_ERR_INVALID, "join: key count must be 1..fields of both inputs");
  for (uint32_t i = 0; i < keycount; ++i)
    if (l->widths[i] != r->widths[i]) return p->fail(RFX_ERR_INVALID, "join: key field widths differ");
  Rel d;
  d.widths = l->widths;
  d.widths.insert(d.widths.end(), r->widths.begin() + keycount, r->widths.end());
  const uint32_t lb = container(total_bits(l->widths)), rb = container(total_bits(r->widths)),
                 db = container(total_bits(d.widths));
  auto ok = [](uint32_t c) { return c == 4 || c == 8 || c == 16; };
  if (!ok(lb) || !ok(rb) || !ok(db))
    return p->fail(RFX_ERR_UNSUPPORTED, "join: inputs and output must be 17..128-bit tuples");
  if (l->sorted < keycount) p->sort_on(a, *l, keycount);
  if (r->sorted < keycount) p->sort_on(b, *r, keycount);
  uint32_t lv = 0, rv = 0;
  for (size_t i = keycount; i < l->widths.size(); ++i) lv += l->widths[i];
  for (size_t i = keycount; i < r->widths.size(); ++i) rv += r->widths[i];
  POp o;
  o.kv = {{"op", q("join")},           {"left", q(a)}, {"right", q(b)}, {"out", q(dest)},
          {"left_value_bits", std::to_string(lv)}, {"right_value_bits", std::to_string(rv)}};
  p->ops.push_back(o);
  // rows come in left order (matches in right order): sorted as far as the left input is
  d.sorted = l->sorted > keycount ? l->sorted : keycount;
  p->define(dest, d);
  return RFX_OK;
}

rfx_status rfx_plan_agg(rfx_plan* p, const char* dest, const char* src, const uint32_t* domains, uint32_t ndomains,
                        uint32_t tag, uint32_t field) {
  if (!p || !domains || ndomains == 0 || ndomains > 16) return RFX_ERR_INVALID;
  if (tag != RFX_AGG_COUNT && tag != RFX_AGG_TOTAL) return p->fail(RFX_ERR_UNSUPPORTED, "agg: COUNT or TOTAL");
  Rel* s = p->rel(src);
  if (!s) return p->fail(RFX_ERR_INVALID, std::string("agg: unknown relation ") + (src ? src : ""));
  if (!p->fresh(dest)) return p->fail(RFX_ERR_INVALID, "agg: destination name in use or empty");
  const uint32_t nf = (uint32_t)s->widths.size();
  std::vector<uint32_t> dom(domains, domains + ndomains);
  uint32_t key_bits = 0;
  for (uint32_t f : dom) {
    if (f >= nf) return p->fail(RFX_ERR_INVALID, "agg: domain field out of range");
    key_bits += s->widths[f];
  }
  if (tag == RFX_AGG_TOTAL && field >= nf) return p->fail(RFX_ERR_INVALID, "agg: summed field out of range");
  const uint32_t vbits_out = tag == RFX_AGG_TOTAL ? 64u : 32u;
  const uint32_t kbytes = key_bits <= 32 ? 4u : key_bits <= 64 ? 8u : key_bits <= 128 ? 16u : 0u;
  Rel d;
  for (uint32_t f : dom) d.widths.push_back(s->widths[f]);
  d.widths.push_back(vbits_out);
  const uint32_t db = container(total_bits(d.widths));
  if (!kbytes || !(db == 4 || db == 8 || db == 16))
    return p->fail(RFX_ERR_UNSUPPORTED, "agg: key plus value must fit 128 bits");
  d.sorted = (uint32_t)d.widths.size();  // sorted by key; one row per key
  const std::string dn(dest);

  // an earlier reduce over the same rows and domains
  for (AggShare& sh : p->shares) {
    if (sh.src != src || sh.version != s->version || sh.domains != dom) continue;
    if (tag == RFX_AGG_TOTAL && sh.total_field != (int)field) continue;
    POp& red = p->ops[sh.reduce_op];
    std::string vcol;
    if (tag == RFX_AGG_COUNT) {
      if (sh.counts.empty()) {
        sh.counts = dn + "#counts";
        red.set("counts", q(sh.counts));
        p->vars[sh.counts] = 4;
      }
      vcol = sh.counts;
    } else {
      vcol = sh.sums;
    }
    POp m;
    m.kv = {{"op", q("merge")}, {"keys", q(sh.keys)}, {"values", q(vcol)}, {"out", q(dn)},
            {"value_bits", std::to_string(vbits_out)}};
    p->ops.push_back(m);
    p->define(dn, d);
    return RFX_OK;
  }

  // the reduce input: s itself when the domains are its leading fields, else a projection
  bool prefix = true;
  for (uint32_t i = 0; i < ndomains; ++i) prefix = prefix && dom[i] == i;
  std::string in = src;
  Rel* t = s;
  uint32_t key_shift = 0, value_shift = 0, value_bits = 1;
  if (prefix) {
    for (uint32_t i = ndomains; i < nf; ++i) key_shift += s->widths[i];
    if (tag == RFX_AGG_TOTAL) {
      if (field < ndomains) prefix = false;  // summing a key field: project it out first
      for (uint32_t i = field + 1; i < nf; ++i) value_shift += s->widths[i];
      value_bits = s->widths[field];
    }
  }
  if (!prefix) {
    std::vector<uint32_t> keep = dom;
    if (tag == RFX_AGG_TOTAL) keep.push_back(field);
    in = dn + "#proj";
    if (rfx_plan_project(p, in.c_str(), src, keep.data(), (uint32_t)keep.size()) != RFX_OK) return RFX_ERR_INVALID;
    t = p->rel(in.c_str());
    s = p->rel(src);
    key_shift = tag == RFX_AGG_TOTAL ? t->widths.back() : 0u;
    value_shift = 0;
    value_bits = tag == RFX_AGG_TOTAL ? t->widths.back() : 1u;
  }
  const uint32_t tb = container(total_bits(t->widths));
  if (!(tb == 4 || tb == 8 || tb == 16)) return p->fail(RFX_ERR_UNSUPPORTED, "agg: input rows must be 17..128 bits");
  if (t->sorted < ndomains) p->sort_on(in, *t, ndomains);
  AggShare sh;
  sh.src = src;
  sh.version = p->rel(src)->version;
  sh.domains = dom;
  sh.total_field = tag == RFX_AGG_TOTAL ? (int)field : -1;
  sh.keys = dn + "#keys";
  p->vars[sh.keys] = kbytes;
  POp red;
  red.kv = {{"op", q("reduce")},
            {"in", q(in)},
            {"key_shift", std::to_string(key_shift)},
            {"value_shift", std::to_string(value_shift)},
            {"value_bits", std::to_string(value_bits)},
            {"keys", q(sh.keys)}};
  if (tag == RFX_AGG_TOTAL) {
    sh.sums = dn + "#sums";
    p->vars[sh.sums] = 8;
    red.set("sums", q(sh.sums));
  } else {
    sh.counts = dn + "#counts";
    p->vars[sh.counts] = 4;
    red.set("counts", q(sh.counts));
  }
  p->ops.push_back(red);
  sh.reduce_op = p->ops.size() - 1;
  POp m;
  m.kv = {{"op", q("merge")},
          {"keys", q(sh.keys)},
          {"values", q(tag == RFX_AGG_TOTAL ? sh.sums : sh.counts)},
          {"out", q(dn)},
          {"value_bits", std::to_string(vbits_out)}};
  p->ops.push_back(m);
  p->shares.push_back(sh);
  p->define(dn, d);
  return RFX_OK;
}

rfx_status rfx_plan_set(rfx_plan* p, const char* dest, const char* a, const char* b, uint32_t kind) {
  if (!p) return RFX_ERR_INVALID;
  static const char* kinds[] = {"union", "difference", "intersection"};
  if (kind > 2) return p->fail(RFX_ERR_INVALID, "set: kind is RFX_SET_UNION, _DIFFERENCE or _INTERSECTION");
  Rel* l = p->rel(a);
  Rel* r = p->rel(b);
  if (!l || !r) return p->fail(RFX_ERR_INVALID, "set: unknown relation");
  if (!p->fresh(dest)) return p->fail(RFX_ERR_INVALID, "set: destination name in use or empty");
  if (l->widths != r->widths) return p->fail(RFX_ERR_INVALID, "set: the relations' fields differ");
  const uint32_t e = container(total_bits(l->widths));
  if (e > 16) return p->fail(RFX_ERR_UNSUPPORTED, "set: tuples wider than 128 bits");
  const uint32_t nf = (uint32_t)l->widths.size();
  if (l->sorted < nf) p->sort_on(a, *l, nf);
  if (r->sorted < nf) p->sort_on(b, *r, nf);
  POp o;
  o.kv = {{"op", q("set")}, {"kind", q(kinds[kind])}, {"a", q(a)}, {"b", q(b)}, {"out", q(dest)}};
  p->ops.push_back(o);
  Rel d;
  d.widths = l->widths;
  d.sorted = nf;
  p->define(dest, d);
  return RFX_OK;
}

rfx_status rfx_plan_unique(rfx_plan* p, const char* name) {
  if (!p) return RFX_ERR_INVALID;
  Rel* r = p->rel(name);
  if (!r) return p->fail(RFX_ERR_INVALID, "unique: unknown relation");
  const uint32_t nf = (uint32_t)r->widths.size();
  if (container(total_bits(r->widths)) > 16) return p->fail(RFX_ERR_UNSUPPORTED, "unique: tuples wider than 128 bits");
  if (r->sorted < nf) p->sort_on(name, *r, nf);
  POp o;
  o.kv = {{"op", q("unique")}, {"rel", q(name)}};
  p->ops.push_back(o);
  ++r->version;
  return RFX_OK;
}

rfx_status rfx_plan_output(rfx_plan* p, const char* name) {
  if (!p) return RFX_ERR_INVALID;
  if (!p->rel(name)) return p->fail(RFX_ERR_INVALID, std::string("output: unknown relation ") + (name ? name : ""));
  for (const auto& o : p->outputs)
    if (o == name) return RFX_OK;
  p->outputs.push_back(name);
  return RFX_OK;
}

size_t rfx_plan_json(rfx_plan* p, char* buf, size_t cap) {
  if (!p) return 0;
  // select -> project fusion: a select whose output only one project reads (and that is
  // not a plan output) becomes one select_project
  std::vector<POp> ops = p->ops;
  std::vector<bool> drop(ops.size(), false);
  auto reads = [](const POp& o, const std::string& n) {
    for (const char* k : {"in", "left", "right", "a", "b", "rel", "keys", "values"}) {
      const std::string* v = o.get(k);
      if (v && *v == q(n)) return true;
    }
    return false;
  };
  for (size_t i = 0; i < ops.size(); ++i) {
    if (*ops[i].get("op") != q("select")) continue;
    const std::string out = ops[i].get("out")->substr(1, ops[i].get("out")->size() - 2);
    bool is_output = false;
    for (const auto& o : p->outputs) is_output = is_output || o == out;
    if (is_output) continue;
    size_t reader = 0, nread = 0;
    for (size_t j = i + 1; j < ops.size(); ++j)
      if (reads(ops[j], out)) {
        ++nread;
        reader = j;
      }
    if (nread != 1 || *ops[reader].get("op") != q("project")) continue;
    // the select's input must not be reordered in place between the two
    bool moved = false;
    for (size_t k = i + 1; k < reader; ++k) {
      const std::string* r = ops[k].get("rel");
      moved = moved || (r && *r == *ops[i].get("in"));
    }
    if (moved) continue;
    POp f;
    f.kv = {{"op", q("select_project")}, {"in", *ops[i].get("in")}, {"out", *ops[reader].get("out")},
            {"widths", *ops[i].get("widths")}, {"cmps", *ops[i].get("cmps")},
            {"out_widths", *ops[reader].get("out_widths")}, {"map", *ops[reader].get("map")}};
    ops[reader] = f;
    drop[i] = true;
  }
  std::string js = "{\"variables\": {";
  bool first = true;
  for (const auto& kv : p->vars) {
    bool used = false;
    for (size_t i = 0; i < ops.size() && !used; ++i)
      if (!drop[i]) {
        used = reads(ops[i], kv.first);
        const std::string* o = ops[i].get("out");
        used = used || (o && *o == q(kv.first));
        for (const char* k : {"keys", "sums", "counts"}) {
          const std::string* v = ops[i].get(k);
          used = used || (v && *v == q(kv.first));
        }
      }
    for (const auto& o : p->outputs) used = used || o == kv.first;
    const Rel* r = p->rel(kv.first.c_str());
    if (!used && !(r && r->input)) continue;
    js += std::string(first ? "" : ", ") + q(kv.first) + ": {\"row_bytes\": " + std::to_string(kv.second) + "}";
    first = false;
  }
  js += "}, \"outputs\": [";
  for (size_t i = 0; i < p->outputs.size(); ++i) js += (i ? ", " : "") + q(p->outputs[i]);
  js += "], \"ops\": [";
  first = true;
  for (size_t i = 0; i < ops.size(); ++i) {
    if (drop[i]) continue;
    js += first ? "\n  {" : ",\n  {";
    first = false;
    for (size_t k = 0; k < ops[i].kv.size(); ++k)
      js += (k ? ", " : "") + q(ops[i].kv[k].first) + ": " + ops[i].kv[k].second;
    js += "}";
  }
  js += "]}";
  if (buf && cap) {
    const size_t m = js.size() < cap - 1 ? js.size() : cap - 1;
    std::memcpy(buf, js.data(), m);
    buf[m] = 0;
  }
  return js.size() + 1;
}

// Field widths and sortedness of a relation of the plan (for callers that read outputs).
rfx_status rfx_plan_schema(const rfx_plan* p, const char* name, uint32_t* widths, uint32_t* nfields,
                           uint32_t* sorted_fields) {
  if (!p || !name || !nfields) return RFX_ERR_INVALID;
  auto it = p->rels.find(name);
  if (it == p->rels.end()) return RFX_ERR_INVALID;
  const Rel& r = it->second;
  if (widths)
    for (size_t i = 0; i < r.widths.size() && i < 16; ++i) widths[i] = r.widths[i];
  *nfields = (uint32_t)r.widths.size();
  if (sorted_fields) *sorted_fields = r.sorted;
  return RFX_OK;
}

}  // extern "C"
