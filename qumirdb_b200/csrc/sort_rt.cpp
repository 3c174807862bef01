// sort_rt.cpp — sort entries of the C ABI (qdb_sort_run, top-K).
#include <algorithm>
#include <cstring>

#include "runtime.h"

using namespace qdb;

extern "C" {

qdb_gpu_program* qdb_gpu_compile_sort(const qdb_sort_spec* spec, char* err, size_t err_len) {
    (void)spec;
    const char* msg = "sort programs are not served by this build";
    if (err && err_len) std::snprintf(err, err_len, "%s", msg);
    t_error = msg;
    return nullptr;
}

int64_t qdb_gpu_sort_run(const qdb_gpu_program* program, qdb_rowset* store, int64_t* row_ids, int64_t* work,
                         uint32_t* counts, int64_t n, bool* descs, bool* nulls_firsts, bool do_sort, int64_t start,
                         int64_t limit, qdb_rowset* out) {
    (void)program; (void)store; (void)row_ids; (void)work; (void)counts; (void)n; (void)descs;
    (void)nulls_firsts; (void)do_sort; (void)start; (void)limit; (void)out;
    SetErr("sort programs are not served by this build");
    return -1;
}

int64_t qdb_gpu_top_k_select(const qdb_gpu_program* program, qdb_rowset* store, int64_t* row_ids, int64_t size,
                             int64_t limit) {
    (void)program; (void)store; (void)row_ids; (void)size; (void)limit;
    SetErr("sort programs are not served by this build");
    return -1;
}

}  // extern "C"
