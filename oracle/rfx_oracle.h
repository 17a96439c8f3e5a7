/*
 * rfx_oracle.h -- CPU restatement of Red Fox's relational-algebra kernel library.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA kernels in
 * redfox_b200/: only tests/, __graft_entry__.smoke() and the CPU-baseline leg of
 * bench.py may load it.  The product path never calls it and has no CPU fallback.
 *
 * Every function cites the reference file:line whose semantics it restates (paths are
 * relative to the sidharth87/redfox tree).  Parity is pinned by tests/golden/: the
 * packing fixture TPC-H/data/A, the TestJoin identity self-join, and vectors produced
 * by the reference's own Union.cu / Difference.cu / Unique.cu / Reduce.cu / Sort.cu
 * compiled for the CPU (oracle/Makefile, target `ref`).
 *
 * Element containers are little-endian byte images of the reference's BasicType:
 * 1, 2, 4, 8 bytes for native unsigned ints, 16/32/64 bytes for PackedNBytes<2/4/8>
 * (limb a[0] lowest, compared from the highest limb down, Tuple.h:231-595).
 */
#ifndef RFX_ORACLE_H
#define RFX_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* A tuple descriptor: up to 16 unsigned bit-fields, field 0 in the most significant
 * used bits (Tuple.h:714-741, BitsAfter :697-705). */
typedef struct {
    uint32_t nfields;
    uint32_t widths[16];
} orc_tuple;

/* Comparison codes = nvcc::RelationalAlgebraKernel::Comparison (RelationalAlgebraKernel.h:157-172). */
enum { ORC_EQ = 1, ORC_NE, ORC_SLT, ORC_LT, ORC_SLE, ORC_LE, ORC_SGT, ORC_GT, ORC_SGE, ORC_GE };
/* Operand kinds = ComparisonOperandType (RelationalAlgebraKernel.h:174-180). */
enum { ORC_OPND_CONSTANT = 0, ORC_OPND_VARIABLE = 2 };
/* Data types = DataType (RelationalAlgebraKernel.h:81-95). */
enum { ORC_I8 = 1, ORC_I16, ORC_I32, ORC_I64, ORC_I128 };
/* Arithmetic ops = ArithmeticOp (RelationalAlgebraKernel.h:121-131). */
enum { ORC_ADD = 0, ORC_MUL, ORC_SUB, ORC_DIV, ORC_MOD };
/* Arith node kinds = ArithExpNodeKind (RelationalAlgebraKernel.h:133-138). */
enum { ORC_NODE_OP = 0, ORC_NODE_CONST, ORC_NODE_INDEX };

typedef struct {
    uint32_t op;         /* ORC_EQ .. ORC_GE */
    uint32_t a_kind;     /* ORC_OPND_* */
    uint32_t b_kind;
    uint32_t a_field;
    uint32_t b_field;
    uint32_t value_type; /* ORC_I8..ORC_I64: C type the field is compared as */
    uint64_t a_const;
    uint64_t b_const;
} orc_cmp;

typedef struct {
    uint32_t kind;   /* ORC_NODE_* */
    uint32_t op;     /* ORC_ADD.. for operator nodes */
    uint32_t type;   /* DataType of a constant / index node */
    int32_t left;    /* child node indices (operator nodes) */
    int32_t right;
    uint32_t pad;
    uint64_t value;  /* constant value, or field index for index nodes */
} orc_node;

typedef struct {
    const orc_node* nodes;
    uint32_t nnodes;
    uint32_t root;
    uint32_t dest_type;  /* DataType of the appended field */
    uint32_t dest_bits;  /* width of the appended field */
} orc_arith;

/* ---- packed tuple codec (Tuple.h) ---- */
uint32_t orc_clamp_bits(uint32_t bits);
uint32_t orc_tuple_bits(const orc_tuple* t);
uint32_t orc_tuple_bytes(const orc_tuple* t);
uint32_t orc_field_shift(const orc_tuple* t, uint32_t field);
uint64_t orc_get_bits(const uint8_t* elem, uint32_t ebytes, uint32_t shift, uint32_t width);
void orc_set_bits(uint8_t* elem, uint32_t ebytes, uint32_t shift, uint32_t width, uint64_t v);
uint64_t orc_extract(const uint8_t* elem, const orc_tuple* t, uint32_t field);
void orc_insert(uint8_t* elem, const orc_tuple* t, uint32_t field, uint64_t v);
void orc_pack_rows(uint8_t* out, size_t n, const orc_tuple* t, const uint64_t* const* cols);
void orc_unpack_rows(const uint8_t* in, size_t n, const orc_tuple* t, uint64_t* const* cols);
int orc_compare(const uint8_t* a, const uint8_t* b, uint32_t ebytes);

/* ---- sort (b40cSort.cu:58-1022, ModernGPUSort.cu) ---- */
void orc_sort_pairs(void* keys, void* vals, size_t n, uint32_t kbytes, uint32_t vbytes,
                    uint32_t begin_bit, uint32_t end_bit);
void orc_sort_pairs_mt(void* keys, void* vals, size_t n, uint32_t kbytes, uint32_t vbytes,
                       uint32_t begin_bit, uint32_t end_bit, int threads);

/* ---- join (ModernGPUJoin.cu:109-733, ModernGPUJoin.h:43-200, benchmarkjoin.cu:40-128) ---- */
void orc_find_bounds(int32_t* lower_bound, int32_t* left_count, uint64_t* total,
                     const void* left, size_t nl, const void* right, size_t nr, uint32_t kbytes);
void orc_join_expand(int32_t* left_idx, int32_t* right_idx, uint64_t nout,
                     const int32_t* lower_bound, const int32_t* scan, size_t nl);
void orc_join_gather(void* out, uint32_t obytes, uint64_t nout,
                     const int32_t* left_idx, const int32_t* right_idx,
                     const void* lkey, uint32_t lkbytes, const void* lval, uint32_t lvbytes,
                     uint32_t lv_bits, const void* rval, uint32_t rvbytes, uint32_t rv_bits);
uint64_t orc_join_tuples(void* out, uint32_t obytes, uint64_t cap,
                         const void* left, size_t nl, uint32_t lbytes, uint32_t l_val_bits,
                         const void* right, size_t nr, uint32_t rbytes, uint32_t r_val_bits);
uint64_t orc_join_count_tuples(const void* left, size_t nl, uint32_t lbytes, uint32_t l_val_bits,
                               const void* right, size_t nr, uint32_t rbytes, uint32_t r_val_bits);

/* ---- reduce / count (Reduce.cu:175-1536) ---- */
uint64_t orc_reduce_sum_i64(const void* keys, size_t n, uint32_t kbytes, const int64_t* vals,
                            void* out_keys, int64_t* out_vals);
uint64_t orc_reduce_count(const void* keys, size_t n, uint32_t kbytes, const uint32_t* vals,
                          void* out_keys, uint32_t* out_counts);

/* ---- set operations (Union.cu, Difference.cu, Unique.cu; benchmarksets.cu:95-125) ---- */
uint64_t orc_set_union(void* out, const void* a, size_t na, const void* b, size_t nb, uint32_t ebytes);
uint64_t orc_set_difference(void* out, const void* a, size_t na, const void* b, size_t nb, uint32_t ebytes);
uint64_t orc_set_intersection(void* out, const void* a, size_t na, const void* b, size_t nb, uint32_t ebytes);
uint64_t orc_unique(void* data, size_t n, uint32_t ebytes);

/* ---- select / arith / project (Select.h, RelationalAlgebraKernel.cpp:2001-2150, Project.h) ---- */
int orc_eval_cmp(const uint8_t* row, const orc_tuple* t, const orc_cmp* c);
uint64_t orc_select(void* out, const void* in, size_t n, const orc_tuple* t,
                    const orc_cmp* cmps, uint32_t ncmp);
int orc_arith_eval(const uint8_t* row, const orc_tuple* t, const orc_arith* a, uint64_t* result);
int orc_arith_rows(void* out, const void* in, size_t n, const orc_tuple* t, const orc_arith* a);
void orc_project(void* out, const void* in, size_t n, const orc_tuple* in_t,
                 const orc_tuple* out_t, const uint32_t* map);

/* ---- fused filter / arith / group-by aggregate (composition of the above) ---- */
int64_t orc_filter_aggregate(const void* in, size_t n, const orc_tuple* t,
                             const orc_cmp* cmps, uint32_t ncmp,
                             const orc_arith* ariths, uint32_t narith,
                             const uint32_t* group_fields, uint32_t ngroup,
                             const uint32_t* sum_fields, uint32_t nsum,
                             uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts,
                             uint64_t cap, int threads);

/* ---- seeded synthetic data (identical formulas on the GPU side) ---- */
uint64_t orc_rand(uint64_t seed, uint64_t stream, uint64_t idx);
uint64_t orc_uniform(uint64_t seed, uint64_t stream, uint64_t idx, uint64_t lo, uint64_t hi);
void orc_gen_uniform_u64(uint64_t* out, size_t n, uint64_t seed, uint64_t stream,
                         uint64_t lo, uint64_t hi, int threads);
void orc_zipf_cdf(double* cdf, size_t n, double s);
void orc_gen_zipf_u64(uint64_t* out, size_t n, uint64_t seed, uint64_t stream,
                      const double* cdf, size_t domain, int threads);

/* ---- string keys: string i of a column is the NUL-terminated text at pool + offs[i]
 * (the reference passes device pointers; offsets into one pool stand for them) ---- */
int orc_str_less(const char* a, const char* b);
int orc_str_equal(const char* a, const char* b);
void orc_str_sort(const char* pool, uint64_t* offs, size_t n, void* vals, uint32_t vbytes);
void orc_str_find_bounds(int32_t* lb, int32_t* cnt, uint64_t* total, const char* pool,
                         const uint64_t* loffs, size_t nl, const uint64_t* roffs, size_t nr);
uint64_t orc_str_count(const char* pool, const uint64_t* offs, size_t n, const uint32_t* vals,
                       uint64_t* out_offs, uint32_t* out_sums);
uint64_t orc_str_codes(const char* pool, const uint64_t* offs, size_t n, uint32_t* codes);

/* ---- double values: the reference's sequential thrust folds (sum, minimum) ---- */
uint64_t orc_reduce_f64_seq(const void* keys, size_t n, uint32_t kb, const double* vals,
                            void* out_keys, double* out_vals, int op_min);

#ifdef __cplusplus
}
#endif
#endif
