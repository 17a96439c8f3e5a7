// scan_program.h -- the per-row program that the select / arith / project / aggregate
// kernels interpret.  It is compiled on the host from the reference-shaped descriptors
// (rfx_cmp = ComparisonExpression, rfx_arith = ArithExpNode tree) and passed to the
// kernels as a __grid_constant__ parameter, so every thread walks the same program and
// all branches on it are warp-uniform.
#pragma once

#include <cstdint>

#include "rfx/rfx.h"

namespace rfx {

constexpr int kMaxCmp = 8;
constexpr int kMaxInstr = 64;
constexpr int kMaxExt = 4;    // appended (arith) fields
constexpr int kMaxRegs = 8;   // expression registers per thread
constexpr int kMaxOut = 16;
constexpr int kMaxGroup = 4;
constexpr int kMaxSum = 4;
constexpr int kMaxGroups = 4096;

// Where a field sits in a container of 64-bit little-endian limbs.
struct FieldLoc {
  uint8_t limb;
  uint8_t off;
  uint8_t width;
  uint8_t pad;
};

struct CmpDesc {
  uint8_t op;
  uint8_t a_var;
  uint8_t b_var;
  uint8_t a_field;
  uint8_t b_field;
  uint8_t pad[3];
  uint64_t a_const;
  uint64_t b_const;
  uint64_t tmask;  // mask of the unsigned C type the operands are compared as
};

// Expression instructions.  Values live in 64-bit registers; 32-bit C types are kept
// normalised (int sign-extended, unsigned int zero-extended) so that the usual
// arithmetic conversions to 64-bit types need no extra step.
enum Op : uint8_t {
  OP_FIELD = 0,   // R[dst] = vfield(field) & imm (C-type truncation)
  OP_CONST,       // R[dst] = imm
  OP_ADD64, OP_SUB64, OP_MUL64,
  OP_ADD_S32, OP_SUB_S32, OP_MUL_S32,
  OP_ADD_U32, OP_SUB_U32, OP_MUL_U32,
  OP_DIV_S32, OP_MOD_S32, OP_DIV_U32, OP_MOD_U32,
  OP_DIV_S64, OP_MOD_S64, OP_DIV_U64, OP_MOD_U64,
  OP_STORE_EXT,   // ext[field] = R[a] & imm
};

struct Instr {
  uint8_t op;
  uint8_t dst;
  uint8_t a;
  uint8_t b;
  uint32_t field;
  uint64_t imm;
};

struct ScanProgram {
  uint32_t in_bytes;
  uint32_t nfields;  // input fields; virtual field v >= nfields is ext[v - nfields]
  uint32_t ncmp;
  uint32_t ninstr;
  uint32_t narith;
  FieldLoc in_loc[16];
  CmpDesc cmps[kMaxCmp];
  Instr code[kMaxInstr];
  // projection into the output container
  uint32_t out_bytes;
  uint32_t nout;
  uint8_t out_src[kMaxOut];  // virtual field per output field; 0xff = constant 0
  FieldLoc out_loc[kMaxOut];
  // group-by aggregation
  uint32_t ngroup;
  uint32_t nsum;
  uint32_t ngroups_total;
  uint8_t group_src[kMaxGroup];
  uint32_t group_domain[kMaxGroup];
  uint32_t group_stride[kMaxGroup];
  uint32_t group_bits[kMaxGroup];
  uint8_t sum_src[kMaxSum];
};

// Host side: build programs from the ABI descriptors.  Return RFX_OK or an error.
rfx_status compile_tuple(const rfx_tuple* t, FieldLoc* locs, uint32_t* bytes, uint32_t* bits);
rfx_status compile_scan(ScanProgram* p, const rfx_tuple* in, const rfx_cmp* cmps, uint32_t ncmp,
                        const rfx_arith_expr* ariths, uint32_t narith);
rfx_status compile_projection(ScanProgram* p, const rfx_tuple* out, const uint32_t* map);
rfx_status compile_aggregate(ScanProgram* p, const uint32_t* group_fields,
                             const uint32_t* group_domain, uint32_t ngroup,
                             const uint32_t* sum_fields, uint32_t nsum);

}  // namespace rfx
