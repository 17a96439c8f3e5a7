/*
 * rfx.h -- C ABI of redfox_b200, a B200-native (sm_100a) implementation of the Red Fox
 * relational-algebra kernel library.
 *
 * Every entry point takes plain device pointers, element counts and a CUDA stream
 * (passed as void*), enqueues its kernels and returns without synchronising.  Buffers
 * are owned by the caller.  Entries that need scratch memory take a caller-provided
 * workspace whose size a matching *_workspace() query reports.  Output sizes are written
 * to device-resident uint64 counters, as the reference's kernels write theirs, so whole
 * plans can be captured in CUDA graphs.  Kernels never trap: a bounded wait that gives
 * up or an input outside a declared bound sets the per-device error word, which
 * rfx_device_status() reads.
 *
 * Each declaration names the reference interface it replaces (paths within the
 * sidharth87/redfox tree).
 */
#ifndef RFX_RFX_H
#define RFX_RFX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference aborts on CUDA errors (b40cSort.cu:48-56) and silently
 * ignores unsupported widths (b40cSort.cu:85-800); these entries report instead. */
typedef enum rfx_status {
    RFX_OK = 0,
    RFX_ERR_INVALID = 1,     /* null pointer, bad descriptor or size */
    RFX_ERR_UNSUPPORTED = 2, /* width / type combination not provided */
    RFX_ERR_CAPACITY = 3,    /* output larger than the caller's capacity */
    RFX_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up */
    RFX_ERR_CUDA = 5,        /* CUDA runtime error */
    RFX_ERR_WORKSPACE = 6    /* workspace smaller than the *_workspace() size */
} rfx_status;

/* Data type codes = nvcc::RelationalAlgebraKernel::DataType
 * (redfox/nvcc/interface/RelationalAlgebraKernel.h:81-95). */
enum { RFX_I8 = 1, RFX_I16 = 2, RFX_I32 = 3, RFX_I64 = 4, RFX_I128 = 5, RFX_I256 = 6, RFX_I512 = 7 };

/* Comparison codes = RelationalAlgebraKernel::Comparison (RelationalAlgebraKernel.h:157-172). */
enum { RFX_EQ = 1, RFX_NE, RFX_SLT, RFX_LT, RFX_SLE, RFX_LE, RFX_SGT, RFX_GT, RFX_SGE, RFX_GE };
/* Operand kinds = ComparisonOperandType (RelationalAlgebraKernel.h:174-180). */
enum { RFX_OPND_CONSTANT = 0, RFX_OPND_VARIABLE = 2 };
/* Arithmetic = ArithmeticOp and ArithExpNodeKind (RelationalAlgebraKernel.h:121-138). */
enum { RFX_ADD = 0, RFX_MUL, RFX_SUB, RFX_DIV, RFX_MOD };
enum { RFX_NODE_OP = 0, RFX_NODE_CONST, RFX_NODE_INDEX };

/* A packed tuple type: up to 16 unsigned bit-fields, field 0 in the most significant used
 * bits, stored in a container of 1/2/4/8/16/32/64 bytes (ra::tuple::Tuple, Tuple.h:714-741;
 * BasicTypeWithBits / PackedNBytes, Tuple.h:231-672). */
typedef struct rfx_tuple {
    uint32_t nfields;
    uint32_t widths[16];
} rfx_tuple;

/* One ANDed comparison of a ComparisonVector (RelationalAlgebraKernel.h:182-208):
 * field-vs-constant or field-vs-field, compared as the unsigned C type `value_type`. */
typedef struct rfx_cmp {
    uint32_t op;
    uint32_t a_kind, b_kind;
    uint32_t a_field, b_field;
    uint32_t value_type;
    uint64_t a_const, b_const;
} rfx_cmp;

/* An ArithExpNode (RelationalAlgebraKernel.h:140-149) in array form. */
typedef struct rfx_arith_node {
    uint32_t kind;
    uint32_t op;
    uint32_t type;
    int32_t left, right;
    uint32_t pad;
    uint64_t value; /* constant, or field index */
} rfx_arith_node;

/* set_arith (RelationalAlgebraKernel.cpp:2001-2150): appends one field computed by an
 * expression tree over the tuple's fields with C integer semantics. */
typedef struct rfx_arith_expr {
    const rfx_arith_node* nodes; /* host memory, read at call time */
    uint32_t nnodes;
    uint32_t root;
    uint32_t dest_type;
    uint32_t dest_bits;
} rfx_arith_expr;

/* ---------------------------------------------------------------- device status */
/* Reads and clears the error word of the current device after synchronising `stream`. */
rfx_status rfx_device_status(void* stream);
/* Library version string. */
const char* rfx_version(void);

/* ---------------------------------------------------------------- select / project */
/* Workspace for the compaction entries below (tile status words). */
size_t rfx_select_workspace(uint64_t n, const rfx_tuple* in);

/* set_select<id> + scan<id> + select_get_result_size<id> + select_gather<id>
 * (ra/interface/Select.h:30-1127; RelationalAlgebraKernel.cpp:1399-1419, :2302-2593) in
 * one order-preserving pass.  Writes the selected rows to `out` and their count to
 * *d_count. */
rfx_status rfx_select(void* out, uint64_t* d_count, const void* in, uint64_t n,
                      const rfx_tuple* in_type, const rfx_cmp* cmps, uint32_t ncmp,
                      void* workspace, size_t workspace_bytes, void* stream);

/* set_arith<id> (RelationalAlgebraKernel.cpp:2001-2150): out = in << dest_bits with the
 * expression in the new last field. */
rfx_status rfx_arith(void* out, const void* in, uint64_t n, const rfx_tuple* in_type,
                     const rfx_arith_expr* arith, void* stream);

/* set_project<id> = ra::cuda::permute (ra/interface/Project.h:58-121): out field k =
 * in field map[k]; map entries >= 16 give 0. */
rfx_status rfx_project(void* out, const void* in, uint64_t n, const rfx_tuple* in_type,
                       const rfx_tuple* out_type, const uint32_t* map, void* stream);

/* Fused select -> arith* -> project with compaction: the rows passing `cmps` get
 * `narith` appended fields (each may read the earlier ones), then `out_type`'s field k
 * is taken from extended field map[k].  Same rows and order as running the reference's
 * select, arith and project kernels one after another. */
rfx_status rfx_select_project(void* out, uint64_t* d_count, const void* in, uint64_t n,
                              const rfx_tuple* in_type, const rfx_cmp* cmps, uint32_t ncmp,
                              const rfx_arith_expr* ariths, uint32_t narith,
                              const rfx_tuple* out_type, const uint32_t* map,
                              void* workspace, size_t workspace_bytes, void* stream);

/* Fused select -> arith* -> group-by SUM(int64)/COUNT over a small key domain: the plan
 * that addAgg builds from project + sort_pair + reduce + count
 * (RelationalAlgebraCompiler.cpp:7852-8643; Reduce.cu), in one pass over the rows.
 * Group field k (an extended field index) must be < group_domain[k]; the groups are the
 * mixed-radix combinations (at most 4096).  Outputs, for the groups that occur, in
 * ascending packed-key order: out_keys[g] = packed group key (group fields concatenated,
 * first field most significant), out_sums[g * nsum + j], out_counts[g]; *d_groups = the
 * number of groups.  A row outside the declared domains sets RFX_ERR_CAPACITY in the
 * device error word. */
size_t rfx_filter_aggregate_workspace(uint64_t n, const rfx_tuple* in_type,
                                      const uint32_t* group_domain, uint32_t ngroup,
                                      uint32_t nsum);
rfx_status rfx_filter_aggregate(const void* in, uint64_t n, const rfx_tuple* in_type,
                                const rfx_cmp* cmps, uint32_t ncmp,
                                const rfx_arith_expr* ariths, uint32_t narith,
                                const uint32_t* group_fields, const uint32_t* group_domain,
                                uint32_t ngroup, const uint32_t* sum_fields, uint32_t nsum,
                                uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts,
                                uint64_t* d_groups, void* workspace, size_t workspace_bytes,
                                void* stream);

/* ---------------------------------------------------------------- sort */
/* Flag for rfx_sort_pairs: read the digit histogram back and skip digit passes whose
 * digit is constant over the input (synchronises the stream once per 128-bit chunk). */
#define RFX_SORT_SKIP_TRIVIAL 1u

/* Workspace of rfx_sort_pairs: the alternate key/value buffers plus histogram and
 * look-back words. */
size_t rfx_sort_workspace(uint64_t n, uint32_t key_bytes, uint32_t value_bytes,
                          uint32_t begin_bit, uint32_t end_bit);

/* Stable ascending LSD radix sort, in place, of n keys of key_bytes (1/2/4/8/16/32/64)
 * on their bits [begin_bit, end_bit) as an unsigned integer (limb a[0] lowest), moving
 * values of value_bytes (0 = keys only, 1/2/4/8/16) with them.  Replaces
 * redfox::sort_pair / sort_key of b40cSort.cu:58-1022 (LSD, bits [0, key_bits)) and of
 * ModernGPUSort.cu:238-548 (stable merge sort on the whole key): both orders are the
 * unique stable order this produces.  Packed tuples sort by a field range directly
 * (no split into key and value arrays).  n < 2^30. */
rfx_status rfx_sort_pairs(void* keys, void* values, uint64_t n, uint32_t key_bytes,
                          uint32_t value_bytes, uint32_t begin_bit, uint32_t end_bit,
                          uint32_t flags, void* workspace, size_t workspace_bytes, void* stream);

/* rfx_sort_pairs out of place: keys_in (and values_in) sorted into keys (and values), the
 * inputs left as they are (the first digit pass reads them; no copy is made).  Inputs and
 * outputs must not overlap; same workspace as rfx_sort_pairs.  No reference counterpart
 * (the reference's sorts work in place); a plan that must keep its input, such as a
 * replayed batched plan, uses it instead of a copy followed by an in-place sort. */
rfx_status rfx_sort_pairs_from(const void* keys_in, const void* values_in, void* keys, void* values,
                               uint64_t n, uint32_t key_bytes, uint32_t value_bytes,
                               uint32_t begin_bit, uint32_t end_bit, uint32_t flags,
                               void* workspace, size_t workspace_bytes, void* stream);

/* redfox::sort_pair / sort_key of b40cSort.cu:58 / :828 with the reference's argument
 * meaning: the key container follows key_bits (<=8: 1 byte, <=16: 2, <=32: 4, <=64: 8),
 * the value container follows value_type (a DataType code), the sort covers bits
 * [0, key_bits).  Every (bits, type) pair is supported, where the reference silently
 * skips all but a fixed list.  Allocates its scratch and synchronises, as the
 * reference does (default stream). */
rfx_status rfx_b40c_sort_pair(void* keys, void* values, uint64_t n, uint64_t key_bits,
                              uint64_t value_type);
rfx_status rfx_b40c_sort_key(void* keys, uint64_t n, uint64_t bits);

/* redfox::sort_pair / sort_key of ModernGPUSort.cu:238 / :484: key and value containers
 * from DataType codes (keys I8..I512, values I8..I128), whole-key stable order. */
rfx_status rfx_mgpu_sort_pair(void* keys, void* values, uint64_t n, uint64_t key_type,
                              uint64_t value_type);
rfx_status rfx_mgpu_sort_key(void* keys, uint64_t n, uint64_t key_type);

/* ---------------------------------------------------------------- reduce / count */
/* Value kinds of rfx_reduce_by_key. */
enum { RFX_VAL_NONE = 0, RFX_VAL_U32 = 1, RFX_VAL_I64 = 2 };

size_t rfx_reduce_by_key_workspace(uint64_t n);

/* Reduce-by-key over runs of equal keys (thrust::reduce_by_key with equal_to / plus, the
 * body of every Reduce.cu entry: count_* :175-660, total_* :665-1536).  keys: n
 * containers of key_bytes (1/2/4/8/16/32), compared bitwise; values: int64
 * (RFX_VAL_I64, exact int64 sums -- the reference has only double and u32 sums), u32
 * (RFX_VAL_U32, u32 sums as count_* computes them) or none (RFX_VAL_NONE).  Writes, per
 * run in input order, the run key, its sum (out_values, same type as the values; may be
 * NULL) and its length (out_counts, u32; may be NULL), and *d_groups = the number of
 * runs.  If d_n is not NULL the element count is min(n, *d_n), read on the device (n is
 * then the capacity the launch is sized for). */
rfx_status rfx_reduce_by_key(const void* keys, uint64_t n, const uint64_t* d_n, uint32_t key_bytes,
                             const void* values, uint32_t value_kind, void* out_keys,
                             void* out_values, uint32_t* out_counts, uint64_t* d_groups,
                             void* workspace, size_t workspace_bytes, void* stream);

/* Reduce-by-key over packed tuples of row_bytes (4/8/16) sorted on their key fields: the
 * key is the row shifted right by key_shift, the value the value_bits-wide field at
 * value_shift (summed as exact int64).  Per run, in order: the key in out_key_bytes
 * (4/8/16), its sum (out_sums, may be NULL) and length (out_counts, may be NULL);
 * *d_groups = runs.  This is addAgg's split + reduce + count (RelationalAlgebraCompiler.cpp
 * :7852-8643, Reduce.cu) on a join output without the split pass.  Workspace:
 * rfx_reduce_by_key_workspace(n). */
rfx_status rfx_reduce_tuples(const void* rows, uint64_t n, const uint64_t* d_n, uint32_t row_bytes,
                             uint32_t key_shift, uint32_t value_shift, uint32_t value_bits,
                             void* out_keys, uint32_t out_key_bytes, int64_t* out_sums,
                             uint32_t* out_counts, uint64_t* d_groups, void* workspace,
                             size_t workspace_bytes, void* stream);

/* redfox::count_{8,16,32,128,256} (Reduce.cu:175-660, Reduce.h:43-83) with the reference's
 * argument meaning: *key_size / *value_size are device-resident byte counts, read on
 * entry and replaced by the output byte counts; the u32 value column is summed per run.
 * key_bytes = 1, 2, 4, 16 or 32.  Synchronous on the default stream, like the reference. */
rfx_status rfx_count_compat(const void* key_begin, const void* value_begin, void* result_key_begin,
                            void* result_value_begin, uint64_t* key_size, uint64_t* value_size,
                            uint32_t key_bytes);
/* redfox::total_64_32 (Reduce.cu:1138-1215): u64 keys, u32 value sums. */
rfx_status rfx_total_64_32_compat(const void* key_begin, const void* value_begin,
                                  void* result_key_begin, void* result_value_begin,
                                  uint64_t* key_size, uint64_t* value_size);
/* The exact int64 SUM with the same byte-size convention (no reference counterpart: the
 * reference's total_* entries sum doubles). */
rfx_status rfx_total_i64_compat(const void* key_begin, const void* value_begin,
                                void* result_key_begin, void* result_value_begin,
                                uint64_t* key_size, uint64_t* value_size, uint32_t key_bytes);

/* Packs an aggregate's key and value columns into tuples: out[i] = key[i] << value_bits |
 * (value[i] & mask(value_bits)) -- the merge that closes the reference's aggregation
 * (ra::cuda::merge, Split_Merge.h:442-495, as addAgg emits it,
 * RelationalAlgebraCompiler.cpp:8536-8643).  Containers: out and keys 4/8/16 bytes, values
 * 4/8 bytes (unused when value_bits is 0).  If d_n is not NULL the row count is
 * min(n, *d_n), read on the device. */
rfx_status rfx_merge_columns(void* out, uint32_t out_bytes, uint64_t n, const uint64_t* d_n,
                             const void* keys, uint32_t key_bytes, const void* values,
                             uint32_t value_bytes, uint32_t value_bits, void* stream);

/* ---------------------------------------------------------------- plan builder */
/* Lowers relational-algebra operators to an executor plan (rfx_exec_create), as the
 * reference's RelationalAlgebraCompiler does to HIR kernel sequences (addJoin,
 * RelationalAlgebraCompiler.cpp:4466-5227; addAgg, :7852-8643; select, project and set
 * builders), without protobuf and without compiling kernels at run time.  Relations are
 * packed tuples: field widths in bits, field 0 most significant.  Keys of a join are the
 * first keycount fields of both inputs; an input not sorted on the fields an operator needs
 * is sorted in place first (the builder tracks sortedness and sorts once).  A select read
 * only by one project is fused into one select_project.  An aggregation over leading
 * fields reads key and value from the rows directly; a COUNT over the same rows and
 * domains as an earlier TOTAL shares its reduce.  Aggregation results are relations
 * (domains..., value): TOTAL values are exact 64-bit sums, COUNT 32-bit counts.  Calls
 * return RFX_ERR_INVALID / RFX_ERR_UNSUPPORTED with a message in rfx_plan_error. */
enum { RFX_AGG_COUNT = 0, RFX_AGG_TOTAL = 1 };
typedef struct rfx_plan rfx_plan;
rfx_status rfx_plan_create(rfx_plan** out);
void rfx_plan_destroy(rfx_plan* plan);
const char* rfx_plan_error(const rfx_plan* plan);
/* An input relation (bound or loaded by name on the executor) sorted on its first
 * sorted_fields fields. */
rfx_status rfx_plan_relation(rfx_plan* plan, const char* name, const uint32_t* widths,
                             uint32_t nfields, uint32_t sorted_fields);
rfx_status rfx_plan_select(rfx_plan* plan, const char* dest, const char* src,
                           const rfx_cmp* cmps, uint32_t ncmp);
rfx_status rfx_plan_project(rfx_plan* plan, const char* dest, const char* src,
                            const uint32_t* fields, uint32_t nfields);
rfx_status rfx_plan_join(rfx_plan* plan, const char* dest, const char* a, const char* b,
                         uint32_t keycount);
rfx_status rfx_plan_agg(rfx_plan* plan, const char* dest, const char* src,
                        const uint32_t* domains, uint32_t ndomains, uint32_t tag,
                        uint32_t field);
/* kind: RFX_SET_UNION / RFX_SET_DIFFERENCE / RFX_SET_INTERSECTION. */
rfx_status rfx_plan_set(rfx_plan* plan, const char* dest, const char* a, const char* b,
                        uint32_t kind);
/* Removes duplicate tuples of a relation in place. */
rfx_status rfx_plan_unique(rfx_plan* plan, const char* name);
rfx_status rfx_plan_output(rfx_plan* plan, const char* name);
/* The executor plan as JSON into buf (cap bytes, NUL-terminated); returns the size needed. */
size_t rfx_plan_json(rfx_plan* plan, char* buf, size_t cap);
rfx_status rfx_plan_schema(const rfx_plan* plan, const char* name, uint32_t* widths,
                           uint32_t* nfields, uint32_t* sorted_fields);

/* ---------------------------------------------------------------- double values */
/* Operations of rfx_reduce_f64. */
enum { RFX_F64_SUM = 0, RFX_F64_MIN = 1 };

size_t rfx_reduce_f64_workspace(uint64_t n);

/* Reduce-by-key over double values: thrust::reduce_by_key with plus<double>
 * (total_{8,16,32,64,128}_double, Reduce.cu:819-1453) or minimum<double> (min_32_double,
 * :1455-1536).  keys: n containers of key_bytes (1/2/4/8/16, compared bitwise; 0 = one run
 * over all values, thrust::reduce of total_double :976-1015).  Per run in input order:
 * the key (out_keys; unused when key_bytes is 0) and the value; *d_groups = runs.
 * RFX_F64_SUM is the exact sum of the run rounded once to nearest-even (independent of
 * evaluation order; a sequential double sum differs from it by at most its own rounding
 * error).  NaN if a term is NaN or both infinities occur, an infinity if one occurs, -0
 * only when every term is -0.  RFX_F64_MIN is the reference's fold acc = acc < v ? acc : v
 * bit for bit (a later equal element replaces an earlier one; a NaN replaces the
 * accumulator and the next element replaces the NaN).  Stream-ordered; a value whose bits
 * fall more than 2^107 below the largest one makes a second, full-range pass do the work
 * (decided on the device).  n < 2^30. */
rfx_status rfx_reduce_f64(const void* keys, uint64_t n, uint32_t key_bytes, const double* values,
                          uint32_t op, void* out_keys, double* out_values, uint64_t* d_groups,
                          void* workspace, size_t workspace_bytes, void* stream);

/* redfox::total_{8,16,32,64,128}_double (Reduce.cu:819-1453) with the reference's byte-size
 * convention (*key_size / *value_size device byte counts, in and out); key_bytes = 1, 2,
 * 4, 8 or 16.  Synchronous on the default stream. */
rfx_status rfx_total_double_compat(const void* key_begin, const void* value_begin,
                                   void* result_key_begin, void* result_value_begin,
                                   uint64_t* key_size, uint64_t* value_size, uint32_t key_bytes);
/* redfox::total_string_double (Reduce.cu:742-817): string keys (device pointers to
 * NUL-terminated strings, runs of equal content), the first pointer of each run. */
rfx_status rfx_total_string_double_compat(const void* key_begin, const void* value_begin,
                                          void* result_key_begin, void* result_value_begin,
                                          uint64_t* key_size, uint64_t* value_size);
/* redfox::min_32_double (Reduce.cu:1455-1536): u32 keys, minimum<double>. */
rfx_status rfx_min_32_double_compat(const void* key_begin, const void* value_begin,
                                    void* result_key_begin, void* result_value_begin,
                                    uint64_t* key_size, uint64_t* value_size);
/* redfox::total_double(result, begin, end) (Reduce.cu:976-1015): the sum of the doubles
 * in [begin, end) into the device double *result (0.0 when empty). */
rfx_status rfx_sum_double_compat(void* result, const void* begin, const void* end);
/* redfox::max_double (Reduce.cu:1058-1136): the maximum of [begin, end) compared as
 * unsigned 64-bit words with initial value 0, as the reference reduces it, into the device
 * word *result. */
rfx_status rfx_max_double_compat(void* result, const void* begin, const void* end);
/* redfox::count(result, begin, end) (Reduce.cu:1017-1056): the u32 sum (mod 2^32) of the
 * u32 words in [begin, end) into *result. */
rfx_status rfx_count_u32_compat(void* result, const void* begin, const void* end);

/* ---------------------------------------------------------------- join */
size_t rfx_join_find_bounds_workspace(uint64_t nl);

/* redfox::find_bounds_{8,16,32,64,128} (ModernGPUJoin.cu:109-663) in one pass: for each
 * sorted left key, lower_bound[i] = first right index with an equal-or-greater key
 * (SortedSearch), and left_count[i] = the exclusive scan of the equal-key counts
 * (SortedEqualityCount + Scan); *d_total = the number of matches.  Keys are containers
 * of key_bytes (1/2/4/8/16) compared whole, high limb first (ModernGPUJoin.cu:27-39).
 * Both inputs sorted ascending; nl, nr < 2^31 (int32 outputs, as the reference's). */
rfx_status rfx_join_find_bounds(int32_t* lower_bound, int32_t* left_count, uint64_t* d_total,
                                const void* left_keys, uint64_t nl, const void* right_keys,
                                uint64_t nr, uint32_t key_bytes, void* workspace,
                                size_t workspace_bytes, void* stream);

/* redfox::join (ModernGPUJoin.cu:665-733, KernelLeftJoin<Tuning, false>): the (left,
 * right) index pairs of the inner join, left ascending then right ascending.  nout
 * sizes the launch; if d_nout is not NULL the pair count is min(nout, *d_nout). */
rfx_status rfx_join_expand(int32_t* left_idx, int32_t* right_idx, uint64_t nout,
                           const uint64_t* d_nout, const int32_t* lower_bound,
                           const int32_t* left_count_scan, uint64_t nl, void* stream);

/* mgpu_join_gather<id> = redfox::gather_{key_key,key_value,value_key,value_value}
 * (ModernGPUJoin.h:43-200): out[k] = lkey[li] << (lval_bits + rval_bits)
 * | lval[li] << rval_bits | rval[ri]; lval / rval may be NULL (their bits are then 0).
 * Containers of 1..64 bytes. */
rfx_status rfx_join_gather(void* out, uint32_t out_bytes, uint64_t nout, const uint64_t* d_nout,
                           const int32_t* left_idx, const int32_t* right_idx, const void* lkey,
                           uint32_t lkey_bytes, const void* lval, uint32_t lval_bytes,
                           uint32_t lval_bits, const void* rval, uint32_t rval_bytes,
                           uint32_t rval_bits, void* stream);

/* Fused sort-merge join of packed tuples sorted on their key fields: the key of a tuple is
 * the tuple shifted right by its value bits (Tuple.h keeps keys in the high fields).
 * Writes out[k] = (L[i] << right_value_bits) | (R[j] & mask(right_value_bits))
 * (combine<>, Tuple.h:942-955 -- the bytes gather_value_value produces after split +
 * find_bounds + join), for the first min(total, capacity) matches in the reference's
 * order, and *d_count = total.  Containers of 4/8/16 bytes. */
size_t rfx_join_tuples_workspace(uint64_t nl);
rfx_status rfx_join_tuples(void* out, uint32_t out_bytes, uint64_t capacity, uint64_t* d_count,
                           const void* left, uint64_t nl, uint32_t left_bytes,
                           uint32_t left_value_bits, const void* right, uint64_t nr,
                           uint32_t right_bytes, uint32_t right_value_bits, void* workspace,
                           size_t workspace_bytes, void* stream);

/* The expansion half of rfx_join_tuples, reusing the bounds a preceding rfx_join_tuples
 * call (capacity 0 counts only) left in `workspace`: the caller reads *d_count, sizes
 * `out`, then emits -- the reference's find_bounds -> join_get_result_size -> Resize ->
 * join_main + gather sequence (RelationalAlgebraCompiler.cpp:4466-5227). */
rfx_status rfx_join_tuples_emit(void* out, uint32_t out_bytes, uint64_t capacity, const void* left,
                                uint64_t nl, uint32_t left_bytes, const void* right, uint64_t nr,
                                uint32_t right_bytes, uint32_t right_value_bits, void* workspace,
                                size_t workspace_bytes, void* stream);

/* addJoin followed by addAgg on the join key (RelationalAlgebraCompiler.cpp:4466-5227,
 * :7852-8643: join, then reduce_by_key SUM / count over the join output) in one operator
 * that never writes the join rows.  left / right are packed tuples sorted on their keys
 * (key = tuple >> value bits, as rfx_join_tuples); the value is the value_bits-wide field
 * of the right tuple at value_shift.  Per key present on both sides, in key order:
 * out_keys (out_key_bytes = 4 or 8; the key fields must fit it, higher bits of the right
 * key are dropped as rfx_reduce_tuples drops them), out_sums = the exact
 * int64 sum of the value over that key's join rows, out_counts = the number of join rows
 * (u32); *d_groups = keys written.  The bytes equal rfx_join_tuples + rfx_reduce_tuples
 * over the join output.  Capacity of the outputs: nr.  Workspace:
 * rfx_join_aggregate_workspace(nr, out_key_bytes). */
size_t rfx_join_aggregate_workspace(uint64_t nr, uint32_t out_key_bytes);
rfx_status rfx_join_aggregate(const void* left, uint64_t nl, uint32_t left_bytes,
                              uint32_t left_value_bits, const void* right, uint64_t nr,
                              uint32_t right_bytes, uint32_t right_value_bits, uint32_t value_shift,
                              uint32_t value_bits, void* out_keys, uint32_t out_key_bytes,
                              int64_t* out_sums, uint32_t* out_counts, uint64_t* d_groups,
                              void* workspace, size_t workspace_bytes, void* stream);

/* Range selection of one relation for up to 256 queries in one scan (no counterpart in
 * the reference, which runs one select per query: Select.h:30-114).  For each row in
 * order and each query q < nq in order, if lo[q] <= field < hi[q] (field = bits
 * [field_shift, field_shift + field_width) of the row, width <= 32) the 8-byte row
 * ((key << 8 | q) << val_width) | val is written, key and val being the bit fields
 * (key_shift, key_width) and (val_shift, val_width) of the input row; key_width + 8 +
 * val_width <= 64.  Input rows of 4/8/16 bytes.  Writes the first `capacity` rows and
 * *d_count = all matches.  lo / hi are host arrays of nq bounds.  Workspace:
 * rfx_multi_select_workspace(n). */
size_t rfx_multi_select_workspace(uint64_t n);
rfx_status rfx_multi_select(void* out, uint64_t capacity, uint64_t* d_count, const void* in,
                            uint64_t n, uint32_t in_bytes, uint32_t field_shift,
                            uint32_t field_width, const uint32_t* lo, const uint32_t* hi,
                            uint32_t nq, uint32_t key_shift, uint32_t key_width,
                            uint32_t val_shift, uint32_t val_width, void* workspace,
                            size_t workspace_bytes, void* stream);

/* redfox::find_bounds_* and redfox::join with the reference's argument meaning (element
 * counts; *result_size on the device).  Own their scratch, synchronous (default
 * stream), as the reference. */
rfx_status rfx_find_bounds_compat(int32_t* lower_bound, int32_t* left_count,
                                  uint64_t* result_size, const void* left_key,
                                  uint64_t left_size, const void* right_key,
                                  uint64_t right_size, uint32_t key_bytes);
rfx_status rfx_join_compat(int32_t* left_indices, int32_t* right_indices, uint64_t result_size,
                           const int32_t* lower_bound, const int32_t* left_count,
                           uint64_t input_size);

/* ---------------------------------------------------------------- set operations */
enum { RFX_SET_UNION = 0, RFX_SET_DIFFERENCE = 1, RFX_SET_INTERSECTION = 2 };

size_t rfx_set_op_workspace(uint32_t op, uint64_t na, uint64_t nb, uint32_t elem_bytes);

/* Multiset set operations on sorted arrays of elem_bytes (1/2/4/8/16) containers, with
 * thrust / STL semantics: union keeps max(m, n) copies of a value (redfox::set_union,
 * Union.cu:47-148), difference max(m - n, 0) (redfox::difference, Difference.cu:35-143),
 * intersection min(m, n) (no reference entry: RelationalAlgebraKernel.cpp:919-922).
 * Output sorted; *d_count = its element count. */
rfx_status rfx_set_op(uint32_t op, void* out, uint64_t* d_count, const void* a, uint64_t na,
                      const void* b, uint64_t nb, uint32_t elem_bytes, void* workspace,
                      size_t workspace_bytes, void* stream);

/* redfox::unique (Unique.cu:36-114): keeps the first of each run of equal elements, in
 * place; *d_count = elements kept. */
size_t rfx_unique_workspace(uint64_t n, uint32_t elem_bytes);
rfx_status rfx_unique(void* data, uint64_t n, uint64_t* d_count, uint32_t elem_bytes,
                      void* workspace, size_t workspace_bytes, void* stream);

/* The reference's set entries with its argument meaning: [lbegin, lend) and [rbegin,
 * rend) device ranges, DataType `type` (I8..I128; I8..I64 for unique), *size = output
 * bytes on the device (for unique: input bytes in, output bytes out).  Synchronous.
 * An unknown type returns RFX_ERR_UNSUPPORTED and leaves the outputs untouched, where the
 * reference falls through to its I8 case (Union.cu:59, Difference.cu:47). */
rfx_status rfx_set_union_compat(void* result, uint64_t* size, void* lbegin, void* lend,
                                void* rbegin, void* rend, uint32_t type);
rfx_status rfx_difference_compat(void* result, uint64_t* size, void* lbegin, void* lend,
                                 void* rbegin, void* rend, uint32_t type);
rfx_status rfx_intersection_compat(void* result, uint64_t* size, void* lbegin, void* lend,
                                   void* rbegin, void* rend, uint32_t type);
rfx_status rfx_unique_compat(void* begin, uint64_t* size, uint64_t type);

/* ---------------------------------------------------------------- string keys */
/* A string column is n 64-bit device pointers to NUL-terminated strings.  Order is the
 * reference's compare_sort_string / compare_string2 (ModernGPUSort.cu:44-67,
 * ModernGPUJoin.cu:72-98): lexicographic on signed char, a proper prefix first.  Equality
 * is compare_string's (Reduce.cu:30-51): the same characters.  No string is read past its
 * terminator.  n < 2^30. */

/* Dictionary codes of a string column: codes[i] = the rank of element i's string among
 * the column's distinct strings (may be NULL), perm[k] = the element at position k of the
 * stable sorted order (may be NULL), *ndistinct (host; may be NULL) = distinct strings.
 * Returns after `stream` has drained. */
rfx_status rfx_string_codes(const void* ptrs, uint64_t n, uint32_t* codes, uint32_t* perm,
                            uint64_t* ndistinct, void* stream);

/* redfox::sort_string_key / sort_string_pair (ModernGPUSort.cu:148-470) and
 * redfox::sort_string (Sort.cu:176-195): stable sort of the pointer column by string,
 * values (value_type I8..I512; 0 = none) moved with their keys.  Synchronous on the
 * default stream. */
rfx_status rfx_sort_string_compat(void* keys, void* values, uint64_t n, uint64_t value_type);

/* redfox::find_bounds_string (ModernGPUJoin.cu:213-300): both columns sorted by string;
 * lower bounds, the exclusive scan of equal-string counts and *result_size (device) as
 * rfx_find_bounds_compat. */
rfx_status rfx_find_bounds_string_compat(int32_t* lower_bound, int32_t* left_count,
                                         uint64_t* result_size, const void* left_key,
                                         uint64_t left_size, const void* right_key,
                                         uint64_t right_size);

/* redfox::count_string / total_string_32 (Reduce.cu:424-480, :665-740): runs of
 * consecutive equal strings, per run its first key pointer and the u32 sum of its values;
 * *key_size / *value_size are device-resident byte counts (in and out). */
rfx_status rfx_count_string_compat(const void* key_begin, const void* value_begin,
                                   void* result_key_begin, void* result_value_begin,
                                   uint64_t* key_size, uint64_t* value_size);

/* rfx_filter_aggregate for callers that cannot allocate device memory when they call it:
 * a runtime that has already handed all device memory out by liveness, or a request path
 * that must not touch the allocator.  It has no counterpart in the reference.  The
 * arguments and outputs are rfx_filter_aggregate's minus the workspace; its scratch is a
 * fixed array inside the library (about 160 KiB, held by every GPU that loads the library
 * until exit), so it allocates nothing.
 * Limits: the array holds 4096 groups x (4 sums + a count), the largest plan
 * rfx_filter_aggregate accepts; plans are validated as that entry validates them and a
 * plan beyond its limits gets the same status (RFX_ERR_UNSUPPORTED).  The first call on a
 * device looks the array's address up; make it before any stream capture.  No call may
 * follow a cudaDeviceReset of that device (the address looked up before it is stale).
 * All calls share the array: calls whose kernels overlap on the GPU race (order them on
 * one stream).  A row outside the declared group domains is recorded as
 * RFX_ERR_CAPACITY in *d_error (a device word the caller zeroes; may be NULL), not in
 * the library's error word. */
rfx_status rfx_filter_aggregate_noalloc(const void* in, uint64_t n, const rfx_tuple* in_type,
                                        const rfx_cmp* cmps, uint32_t ncmp,
                                        const rfx_arith_expr* ariths, uint32_t narith,
                                        const uint32_t* group_fields, const uint32_t* group_domain,
                                        uint32_t ngroup, const uint32_t* sum_fields, uint32_t nsum,
                                        uint64_t* out_keys, int64_t* out_sums, uint64_t* out_counts,
                                        uint64_t* d_groups, uint32_t* d_error, void* stream);

/* ---------------------------------------------------------------- synthetic data */
/* Column j of row i = lo[j] + mulhi64(rand(seed, stream_j, i), hi[j] - lo[j]) with the
 * SplitMix64 stream below, packed as `type`.  The generator behind the benchmarks. */
rfx_status rfx_gen_uniform_rows(void* out, uint64_t n, const rfx_tuple* type, uint64_t seed,
                                const uint64_t* lo, const uint64_t* hi, void* stream);

/* ---------------------------------------------------------------- autotuning
 * No counterpart in the reference (its kernels have fixed launch shapes).  Operators with
 * several compiled variants (the TMA-staged rfx_reduce_tuples: chunked, or a look-back per
 * 256- or 128-line tile; the
 * set filters behind rfx_set_op: 8 or 4 items per thread; the plan-specialised rfx_select /
 * rfx_select_project: items per thread; the plan-specialised rfx_filter_aggregate: rows per
 * thread per iteration) run their default unless tuning is on.  With
 * mode 1 (or RFX_TUNE=1 in the environment) the first call of each (operator, shape, size
 * class of 4x in n) times every variant on the caller's inputs and stream (CUDA events,
 * best of three after one untimed run, synchronising the stream) and later calls of that
 * class run the fastest.  Do not enable it while capturing a stream into a graph. */
void rfx_tune_set(int mode);
void rfx_tune_reset(void);
/* Pins an operator (1 reduce_tuples, 2 set filters, 3 select / project, 4 filter-aggregate)
 * to one variant, ahead of tuning and of the default; a negative variant unpins it. */
void rfx_tune_force(uint32_t op, int variant);
/* The tuning table as text lines "op=.. shape=.. class=.. variant=.. ms=t0,t1,..";
 * returns the bytes needed (including the terminating 0); writes at most cap bytes. */
size_t rfx_tune_dump(char* buf, size_t cap);

/* ---------------------------------------------------------------- plan executor
 * The part of Harmony's runtime that runs an RA plan's kernel sequence
 * (harmony/runtime/implementation/Runtime.cpp:295-445): variables allocated at their
 * first definition and freed after their last use, output sizes read back where the next
 * operator is sized by them, inputs loaded from packed relation files
 * (Runtime.cpp:191-206) or bound to caller memory -- with a JSON plan instead of the HIR
 * protobuf (the grammar is in redfox_b200/csrc/exec.cpp).  Device memory comes from the
 * stream-ordered allocator and is held within `budget_bytes` (0: no limit); an operator
 * that would exceed it fails with RFX_ERR_CAPACITY.  No counterpart in the C ABI of the
 * reference (its runtime called the kernel library). */
typedef struct rfx_exec rfx_exec;
rfx_status rfx_exec_create(rfx_exec** out, const char* plan_json, uint64_t budget_bytes, char* err,
                           size_t err_cap);
void rfx_exec_destroy(rfx_exec* exec);
rfx_status rfx_exec_bind(rfx_exec* exec, const char* name, void* device_ptr, uint64_t bytes);
rfx_status rfx_exec_load(rfx_exec* exec, const char* name, const char* path, void* stream);
rfx_status rfx_exec_run(rfx_exec* exec, void* stream);
rfx_status rfx_exec_output(rfx_exec* exec, const char* name, void** device_ptr, uint64_t* rows,
                           uint32_t* row_bytes);
rfx_status rfx_exec_stats(rfx_exec* exec, uint64_t* in_use, uint64_t* peak, uint64_t* ops, char* err,
                          size_t err_cap);
/* Copies a variable's rows (after a run) to caller device memory of cap_bytes. */
rfx_status rfx_exec_copy_out(rfx_exec* exec, const char* name, void* dst, uint64_t cap_bytes, void* stream);

/* The plan as a CUDA graph (Harmony runs a plan's kernels one launch at a time,
 * Runtime.cpp:304-445; here the whole sequence is one graph launch).  rfx_exec_capture
 * runs the plan once eagerly on `stream` (a non-default stream) to learn every size it
 * reads back and every allocation, allocates one arena of that total (against the
 * budget) and captures the op sequence with its memory taken from the arena and the
 * learnt sizes in place of the read-backs.  rfx_exec_replay launches the graph and checks
 * that each intermediate size the graph produced equals the captured one: RFX_OK means
 * the outputs (rfx_exec_output) equal an eager run's; RFX_ERR_CAPACITY means the inputs'
 * contents changed the plan's shape and the plan must run eagerly or be captured again.
 * Inputs must stay bound to the same memory; tuning must be off. */
rfx_status rfx_exec_capture(rfx_exec* exec, void* stream);
rfx_status rfx_exec_replay(rfx_exec* exec, void* stream);

#ifdef __cplusplus
}
#endif
#endif
