// noalloc_rt.cpp — the aggregate entry point that allocates no device memory
// (qdb_gpu_agg_run_noalloc).  Inputs and outputs must already be in device
// memory; table, counters and finalize scratch live in a fixed file-scope
// device array (agg.cu).
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "runtime.h"

using namespace qdb;

extern "C" int64_t qdb_gpu_agg_run_noalloc(const qdb_gpu_program* prog, const qdb_rowset* batch,
                                           qdb_column* out_columns, int64_t out_capacity) {
    t_error.clear();
    if (!prog || prog->kind != PK_AGG || !batch || !out_columns || out_capacity < 0) {
        SetErr("agg_run_noalloc: needs an aggregate program, a row set and output columns");
        return -1;
    }
    const AggLowering& lw = prog->agg;
    AggPlan plan = lw.plan;
    const int64_t n = batch->RowCount;
    // Resolve columns in place: every buffer must already be device memory.
    for (int slot = 0; slot < plan.ncols; ++slot) {
        ColDesc& cd = plan.cols[slot];
        const int input = lw.cols.input_of[slot];
        if (input >= batch->ColumnCount) {
            SetErr("agg_run_noalloc: the row set has too few columns");
            return -1;
        }
        const qdb_column& c = batch->Columns[input];
        if (n > 0 && !IsDevicePtr(c.Data)) {
            SetErr("agg_run_noalloc: column %d is not in device memory (this entry point copies nothing)", input);
            return -1;
        }
        cd.data = c.Data;
        cd.bit_off = prog->columns[input].type == QDB_TYPE_BOOL ? c.DataBitOffset : 0;
        cd.mask = nullptr;
        cd.mask_off = 0;
        if (c.Mask) {
            if (!IsDevicePtr(c.Mask)) {
                SetErr("agg_run_noalloc: the validity mask of column %d is not in device memory", input);
                return -1;
            }
            cd.mask = c.Mask;
            cd.mask_off = c.MaskBitOffset;
        }
    }
    if (batch->Selection && !IsDevicePtr(batch->Selection)) {
        SetErr("agg_run_noalloc: the selection vector is not in device memory");
        return -1;
    }
    plan.selection = batch->Selection;
    plan.has_selection = batch->Selection != nullptr;

    cudaStream_t s = CurStream();
    std::vector<AggOutputCol> cols(size_t(lw.out.n));
    // Every output buffer is checked before anything is written.
    for (int k = 0; k < lw.out.n; ++k) {
        const qdb_column& oc = out_columns[k];
        if (!oc.Data || !IsDevicePtr(oc.Data)) {
            SetErr("agg_run_noalloc: output column %d needs a device buffer", k);
            return -1;
        }
        const int type = lw.out.out_type[k];
        const uintptr_t align = type == QDB_TYPE_DECIMAL128 ? 16 : uintptr_t(std::max(1, StorageWidth(type)));
        if (reinterpret_cast<uintptr_t>(oc.Data) % std::min<uintptr_t>(align, 8)) {
            SetErr("agg_run_noalloc: output column %d is not aligned to its value width", k);
            return -1;
        }
        if (oc.Mask && (!IsDevicePtr(oc.Mask) || reinterpret_cast<uintptr_t>(oc.Mask) % 4)) {
            SetErr("agg_run_noalloc: output mask %d must be 4-byte aligned device memory of "
                   "(out_capacity + 31) / 32 uint32 words", k);
            return -1;
        }
        if (oc.Offsets && type == QDB_TYPE_CHAR1 &&
            (!IsDevicePtr(oc.Offsets) || reinterpret_cast<uintptr_t>(oc.Offsets) % 4)) {
            SetErr("agg_run_noalloc: output offsets %d must be 4-byte aligned device memory", k);
            return -1;
        }
    }
    for (int k = 0; k < lw.out.n; ++k) {
        qdb_column& oc = out_columns[k];
        AggOutputCol& c = cols[size_t(k)];
        std::memset(&c, 0, sizeof(c));
        c.type = lw.out.out_type[k];
        c.data = oc.Data;
        if (oc.Mask) {
            c.valid = reinterpret_cast<uint32_t*>(const_cast<uint8_t*>(oc.Mask));
            cudaMemsetAsync(c.valid, 0, size_t((out_capacity + 31) / 32) * 4, s);
        }
        if (oc.Offsets && c.type == QDB_TYPE_CHAR1) c.offsets = static_cast<int32_t*>(oc.Offsets);
    }
    const bool priv = plan.nkeyparts == 0 || (prog->expected_groups > 0 && prog->expected_groups <= 64);
    std::string err;
    const int64_t groups = AggRunNoAlloc(plan, lw.out, n, cols.data(), int(cols.size()), out_capacity, priv, s, err);
    if (groups < 0) {
        SetErr("agg_run_noalloc: %s", err.c_str());
        return -1;
    }
    return groups;
}
