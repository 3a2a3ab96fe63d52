// C-ABI entry points for the operators (declared in include/aspher_b200.h).
// No exception crosses this boundary: every call returns an int status and
// leaves a message for aspher_last_error().
#include "../../include/aspher_b200.h"
#include "ops.hpp"

#include <cstring>
#include <string>

namespace asb {
thread_local std::string g_last_error;
void set_last_error(const std::string& m) { g_last_error = m; }
}  // namespace asb

struct aspher_op {
    asb::Operator* impl;
};

#define ASB_API_BEGIN try {
#define ASB_API_END                                               \
    }                                                             \
    catch (const asb::Error& e) {                                 \
        asb::set_last_error(e.what());                            \
        return e.code;                                            \
    }                                                             \
    catch (const std::exception& e) {                             \
        asb::set_last_error(e.what());                            \
        return ASPHER_ECUDA;                                      \
    }                                                             \
    catch (...) {                                                 \
        asb::set_last_error("unknown error");                     \
        return ASPHER_ECUDA;                                      \
    }

extern "C" {

int aspher_abi_version(void) { return ASPHER_B200_ABI_VERSION; }

const char* aspher_last_error(void) { return asb::g_last_error.c_str(); }

int64_t aspher_launch_count(void) { return (int64_t)asb::launch_count(); }

int aspher_op_create_ex(int backend, int grid_size, double domain_size, double E_star,
                        int flags, aspher_op** out) {
    ASB_API_BEGIN
    if (!out) throw asb::Error(ASPHER_EINVAL, "aspher_op_create: out is NULL");
    *out = nullptr;
    if (backend != ASPHER_BACKEND_FFT && backend != ASPHER_BACKEND_PERIODIC)
        throw asb::Error(ASPHER_EINVAL, "unknown backend (expected fft or periodic)");
    static_assert(ASPHER_OPF_SPLIT_COLUMNS == asb::OPF_SPLIT_COLUMNS &&
                      ASPHER_OPF_SPLIT_KH == asb::OPF_SPLIT_KH,
                  "flag values of the ABI and the operator agree");
    auto* op = new aspher_op{nullptr};
    try {
        op->impl = new asb::Operator(backend, grid_size, domain_size, E_star, flags);
    } catch (...) {
        delete op;
        throw;
    }
    *out = op;
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_create(int backend, int grid_size, double domain_size, double E_star,
                     aspher_op** out) {
    return aspher_op_create_ex(backend, grid_size, domain_size, E_star, 0, out);
}

int aspher_op_destroy(aspher_op* op) {
    ASB_API_BEGIN
    if (!op) return ASPHER_OK;
    delete op->impl;
    delete op;
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_matvec(aspher_op* op, int dtype, const void* x, void* y, void* stream) {
    ASB_API_BEGIN
    if (!op || !op->impl) throw asb::Error(ASPHER_EINVAL, "aspher_op_matvec: NULL operator");
    if (!x || !y) throw asb::Error(ASPHER_EINVAL, "aspher_op_matvec: NULL buffer");
    if (dtype != ASPHER_F32 && dtype != ASPHER_F64)
        throw asb::Error(ASPHER_EINVAL, "aspher_op_matvec: dtype must be F32 or F64");
    const size_t align = dtype == ASPHER_F64 ? 16 : 8;
    if (((uintptr_t)x % align) || ((uintptr_t)y % align))
        throw asb::Error(ASPHER_EINVAL, "aspher_op_matvec: buffers must be 16-byte aligned");
    op->impl->apply_caller(dtype == ASPHER_F64, x, y, static_cast<cudaStream_t>(stream));
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_get_info(const aspher_op* op, aspher_op_info* info) {
    ASB_API_BEGIN
    if (!op || !op->impl || !info) throw asb::Error(ASPHER_EINVAL, "aspher_op_get_info: NULL");
    const asb::Operator& o = *op->impl;
    std::memset(info, 0, sizeof(*info));
    info->backend = o.backend;
    info->grid_size = o.Nl;
    // the transform side of the compute pipeline (embedded grids: that of
    // the power-of-two grid the caller's block sits in)
    info->padded_side = o.kind == asb::OP_FFT ? 2 * o.Ns : o.Ns;
    info->n = (int64_t)o.Nl * o.Nl;
    if (o.kind == asb::OP_FFT)
        info->bytes_spectrum = (int64_t)(o.Ns + 16) * (o.Ns + 1) * 12 + (int64_t)(o.Ns + 1) * (o.Ns + 1) * 8;
    else  // the periodic multiplier tables (FP32, and FP64 where FP64 applies exist)
        info->bytes_spectrum = (int64_t)(o.Ns / 2 + 16) * (o.Ns / 2 + 1) * (o.psym_d ? 12 : 4);
    info->bytes_scratch = (int64_t)(o.spec_d_bytes + o.spec_f_bytes);
    info->bytes_total = (int64_t)o.resident_bytes();
    info->max_im_ratio = o.max_im_ratio;
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_set_variants(aspher_op* op, int dtype, int row_variant, int col_variant) {
    ASB_API_BEGIN
    if (!op || !op->impl) throw asb::Error(ASPHER_EINVAL, "aspher_op_set_variants: NULL operator");
    op->impl->set_variants(dtype == ASPHER_F64, row_variant, col_variant);
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_get_variants(const aspher_op* op, int dtype, int* row_variant, int* col_variant,
                           int* col_tile) {
    ASB_API_BEGIN
    if (!op || !op->impl) throw asb::Error(ASPHER_EINVAL, "aspher_op_get_variants: NULL operator");
    const int d = dtype == ASPHER_F64;
    if (row_variant) *row_variant = op->impl->rowv[d];
    if (col_variant) *col_variant = op->impl->colv[d];
    if (col_tile) *col_tile = op->impl->ct[d];
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_autotune(aspher_op* op, int dtype, int reps, int* row_variant, int* col_variant,
                       double* best_ms) {
    ASB_API_BEGIN
    if (!op || !op->impl) throw asb::Error(ASPHER_EINVAL, "aspher_op_autotune: NULL operator");
    if (reps < 1) throw asb::Error(ASPHER_EINVAL, "aspher_op_autotune: reps must be >= 1");
    int rv = 0, cv = 0;
    const double ms = op->impl->autotune(dtype == ASPHER_F64, reps, rv, cv);
    if (row_variant) *row_variant = rv;
    if (col_variant) *col_variant = cv;
    if (best_ms) *best_ms = ms;
    return ASPHER_OK;
    ASB_API_END
}

int aspher_op_love_table(const aspher_op* op, double* host_out) {
    ASB_API_BEGIN
    if (!op || !op->impl || !host_out) throw asb::Error(ASPHER_EINVAL, "aspher_op_love_table: NULL");
    const asb::Operator& o = *op->impl;
    if (o.backend != asb::OP_FFT || !o.table)
        throw asb::Error(ASPHER_EINVAL, "aspher_op_love_table: only the fft backend has a table");
    // the Nl x Nl offsets of the caller's grid (the device table has the
    // compute grid's pitch)
    std::lock_guard<std::recursive_mutex> setup(asb::setup_mutex());
    ASB_CUDA(cudaMemcpy2D(host_out, (size_t)o.Nl * sizeof(double), o.table,
                          (size_t)o.Ns * sizeof(double), (size_t)o.Nl * sizeof(double), o.Nl,
                          cudaMemcpyDeviceToHost));
    return ASPHER_OK;
    ASB_API_END
}

}  // extern "C"
