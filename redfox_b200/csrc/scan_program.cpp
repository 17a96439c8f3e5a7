// scan_program.cpp -- host compiler from reference-shaped descriptors to ScanProgram.
#include "scan_program.h"

#include <cstring>

namespace rfx {

namespace {

uint32_t clamp_bits(uint32_t v) {
  // Clamp<v> (ra/interface/Tuple.h:31-37)
  return v <= 8 ? 8 : v <= 16 ? 16 : v <= 32 ? 32 : v <= 64 ? 64 : v <= 128 ? 128
       : v <= 256 ? 256 : v <= 512 ? 512 : 0;
}

uint64_t type_mask(uint32_t type) {
  switch (type) {
    case RFX_I8: return 0xffull;
    case RFX_I16: return 0xffffull;
    case RFX_I32: return 0xffffffffull;
    case RFX_I64: return ~0ull;
    default: return 0;
  }
}

uint64_t width_mask(uint32_t w) { return w >= 64 ? ~0ull : ((1ull << w) - 1); }

// C types of the generated expression code (RelationalAlgebraKernel.cpp:1822-1939).
enum CType { CT_I32, CT_U32, CT_I64, CT_U64 };

struct Gen {
  ScanProgram* p;
  const rfx_arith_expr* a;
  uint32_t nvfields;
  uint32_t next_reg;
  int depth;
  bool ok;

  bool emit(Instr ins) {
    if (p->ninstr >= (uint32_t)kMaxInstr) return ok = false;
    p->code[p->ninstr++] = ins;
    return true;
  }

  // Returns the register holding the node's value and its C type.
  bool node(uint32_t idx, uint8_t* reg, CType* ct) {
    if (!ok || idx >= a->nnodes || ++depth > 32) return ok = false;
    const rfx_arith_node& nd = a->nodes[idx];
    bool r = true;
    if (nd.kind == RFX_NODE_CONST) {
      if (next_reg >= (uint32_t)kMaxRegs) return ok = false;
      *reg = (uint8_t)next_reg++;
      // a decimal literal is int, then long, then unsigned long
      *ct = nd.value <= 0x7fffffffull ? CT_I32 : nd.value <= 0x7fffffffffffffffull ? CT_I64 : CT_U64;
      Instr ins{OP_CONST, *reg, 0, 0, 0, nd.value};
      r = emit(ins);
    } else if (nd.kind == RFX_NODE_INDEX) {
      if (next_reg >= (uint32_t)kMaxRegs || nd.value >= nvfields) return ok = false;
      *reg = (uint8_t)next_reg++;
      uint64_t m;
      switch (nd.type) {
        case RFX_I8: *ct = CT_I32; m = 0xff; break;      // unsigned char promotes to int
        case RFX_I16: *ct = CT_I32; m = 0xffff; break;   // unsigned short promotes to int
        case RFX_I32: *ct = CT_U32; m = 0xffffffffull; break;
        case RFX_I64: *ct = CT_U64; m = ~0ull; break;
        default: return ok = false;
      }
      Instr ins{OP_FIELD, *reg, 0, 0, (uint32_t)nd.value, m};
      r = emit(ins);
    } else if (nd.kind == RFX_NODE_OP) {
      uint8_t ra, rb;
      CType ca, cb;
      if (nd.left < 0 || nd.right < 0) return ok = false;
      if (!node((uint32_t)nd.left, &ra, &ca) || !node((uint32_t)nd.right, &rb, &cb)) return ok = false;
      bool wide = ca >= CT_I64 || cb >= CT_I64;
      CType c = wide ? ((ca == CT_U64 || cb == CT_U64) ? CT_U64 : CT_I64)
                     : ((ca == CT_U32 || cb == CT_U32) ? CT_U32 : CT_I32);
      uint8_t op;
      switch (nd.op) {
        case RFX_ADD: op = wide ? OP_ADD64 : (c == CT_I32 ? OP_ADD_S32 : OP_ADD_U32); break;
        case RFX_SUB: op = wide ? OP_SUB64 : (c == CT_I32 ? OP_SUB_S32 : OP_SUB_U32); break;
        case RFX_MUL: op = wide ? OP_MUL64 : (c == CT_I32 ? OP_MUL_S32 : OP_MUL_U32); break;
        case RFX_DIV:
          op = wide ? (c == CT_I64 ? OP_DIV_S64 : OP_DIV_U64) : (c == CT_I32 ? OP_DIV_S32 : OP_DIV_U32);
          break;
        case RFX_MOD:
          op = wide ? (c == CT_I64 ? OP_MOD_S64 : OP_MOD_U64) : (c == CT_I32 ? OP_MOD_S32 : OP_MOD_U32);
          break;
        default: return ok = false;
      }
      Instr ins{op, ra, ra, rb, 0, 0};
      r = emit(ins);
      *reg = ra;
      *ct = c;
      next_reg = ra + 1u;  // rb (and anything above) is free again
    } else {
      return ok = false;
    }
    --depth;
    return r && ok;
  }
};

}  // namespace

rfx_status compile_tuple(const rfx_tuple* t, FieldLoc* locs, uint32_t* bytes, uint32_t* bits) {
  if (!t || t->nfields == 0 || t->nfields > 16) return RFX_ERR_INVALID;
  uint32_t total = 0;
  for (uint32_t i = 0; i < t->nfields; ++i) {
    if (t->widths[i] > 64) return RFX_ERR_UNSUPPORTED;
    total += t->widths[i];
  }
  uint32_t c = clamp_bits(total);
  if (c == 0 || total == 0) return RFX_ERR_UNSUPPORTED;
  uint32_t upto = 0;
  for (uint32_t i = 0; i < t->nfields; ++i) {
    upto += t->widths[i];
    uint32_t shift = total - upto;  // BitsAfter (Tuple.h:697-705)
    if (locs) locs[i] = FieldLoc{(uint8_t)(shift / 64), (uint8_t)(shift % 64), (uint8_t)t->widths[i], 0};
  }
  if (bytes) *bytes = c / 8;
  if (bits) *bits = total;
  return RFX_OK;
}

rfx_status compile_scan(ScanProgram* p, const rfx_tuple* in, const rfx_cmp* cmps, uint32_t ncmp,
                        const rfx_arith_expr* ariths, uint32_t narith) {
  std::memset(p, 0, sizeof(*p));
  rfx_status st = compile_tuple(in, p->in_loc, &p->in_bytes, nullptr);
  if (st != RFX_OK) return st;
  p->nfields = in->nfields;
  if (ncmp > (uint32_t)kMaxCmp || narith > (uint32_t)kMaxExt) return RFX_ERR_UNSUPPORTED;
  if ((ncmp && !cmps) || (narith && !ariths)) return RFX_ERR_INVALID;
  p->ncmp = ncmp;
  for (uint32_t i = 0; i < ncmp; ++i) {
    const rfx_cmp& c = cmps[i];
    if (c.op < RFX_EQ || c.op > RFX_GE) return RFX_ERR_UNSUPPORTED;
    CmpDesc& d = p->cmps[i];
    d.op = (uint8_t)c.op;
    d.tmask = type_mask(c.value_type);
    if (!d.tmask) return RFX_ERR_UNSUPPORTED;
    for (int side = 0; side < 2; ++side) {
      uint32_t kind = side ? c.b_kind : c.a_kind;
      uint32_t field = side ? c.b_field : c.a_field;
      uint64_t k = side ? c.b_const : c.a_const;
      if (kind == RFX_OPND_VARIABLE) {
        if (field >= in->nfields) return RFX_ERR_INVALID;
        (side ? d.b_var : d.a_var) = 1;
        (side ? d.b_field : d.a_field) = (uint8_t)field;
      } else if (kind == RFX_OPND_CONSTANT) {
        (side ? d.b_const : d.a_const) = k;
      } else {
        return RFX_ERR_UNSUPPORTED;
      }
    }
  }
  p->narith = narith;
  for (uint32_t j = 0; j < narith; ++j) {
    const rfx_arith_expr& a = ariths[j];
    if (!a.nodes || !a.nnodes || a.dest_bits == 0 || a.dest_bits > 64 || !type_mask(a.dest_type))
      return RFX_ERR_INVALID;
    Gen g{p, &a, in->nfields + j, 0, 0, true};
    uint8_t reg;
    CType ct;
    if (!g.node(a.root, &reg, &ct)) return RFX_ERR_UNSUPPORTED;
    Instr st_ins{OP_STORE_EXT, 0, reg, 0, j, type_mask(a.dest_type) & width_mask(a.dest_bits)};
    if (!g.emit(st_ins)) return RFX_ERR_UNSUPPORTED;
  }
  return RFX_OK;
}

rfx_status compile_projection(ScanProgram* p, const rfx_tuple* out, const uint32_t* map) {
  if (!out || !map) return RFX_ERR_INVALID;
  rfx_status st = compile_tuple(out, p->out_loc, &p->out_bytes, nullptr);
  if (st != RFX_OK) return st;
  p->nout = out->nfields;
  uint32_t nv = p->nfields + p->narith;
  for (uint32_t k = 0; k < out->nfields; ++k) p->out_src[k] = map[k] < nv && map[k] < 16 + (uint32_t)kMaxExt ? (uint8_t)map[k] : 0xff;
  return RFX_OK;
}

rfx_status compile_aggregate(ScanProgram* p, const uint32_t* gf, const uint32_t* gd, uint32_t ngroup,
                             const uint32_t* sf, uint32_t nsum) {
  if (ngroup == 0 || ngroup > (uint32_t)kMaxGroup || nsum > (uint32_t)kMaxSum) return RFX_ERR_UNSUPPORTED;
  if (!gf || !gd || (nsum && !sf)) return RFX_ERR_INVALID;
  uint32_t nv = p->nfields + p->narith;
  uint64_t total = 1;
  uint32_t key_bits = 0;
  p->ngroup = ngroup;
  p->nsum = nsum;
  for (uint32_t k = 0; k < ngroup; ++k) {
    if (gf[k] >= nv || gd[k] == 0) return RFX_ERR_INVALID;
    p->group_src[k] = (uint8_t)gf[k];
    p->group_domain[k] = gd[k];
    total *= gd[k];
    if (total > (uint64_t)kMaxGroups) return RFX_ERR_UNSUPPORTED;
  }
  uint32_t stride = 1;
  for (int k = (int)ngroup - 1; k >= 0; --k) {
    p->group_stride[k] = stride;
    stride *= gd[k];
  }
  for (uint32_t k = 0; k < ngroup; ++k) {
    uint32_t v = gf[k];
    uint32_t w = v < p->nfields ? p->in_loc[v].width : 64;
    if (v >= p->nfields) {
      // the appended field's width is the mask its STORE_EXT applies
      for (uint32_t i = 0; i < p->ninstr; ++i)
        if (p->code[i].op == OP_STORE_EXT && p->code[i].field == v - p->nfields) {
          uint64_t m = p->code[i].imm;
          w = 0;
          while (w < 64 && ((m >> w) & 1)) ++w;
        }
    }
    p->group_bits[k] = w;
    key_bits += w;
  }
  if (key_bits > 64) return RFX_ERR_UNSUPPORTED;
  p->ngroups_total = (uint32_t)total;
  for (uint32_t j = 0; j < nsum; ++j) {
    if (sf[j] >= nv) return RFX_ERR_INVALID;
    p->sum_src[j] = (uint8_t)sf[j];
  }
  return RFX_OK;
}

}  // namespace rfx
