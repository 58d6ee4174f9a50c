// capi.cu -- the extern "C" boundary (include/sparsesolv_b200.h). Every entry
// point converts exceptions into a status code plus a thread-local message.
#include <cstring>
#include <string>

#include "solver_api.hpp"

namespace {

thread_local std::string g_last_error;

template <typename F>
int guarded(F&& f) {
    try {
        f();
        g_last_error.clear();
        return SSV_OK;
    } catch (const ssv::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return SSV_ERR_ALLOC;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return SSV_ERR_RUNTIME;
    }
}

void require_device() {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0)
        ssv::fail(SSV_ERR_NO_DEVICE,
                  "sparsesolv_b200: no CUDA device available (this library has no CPU path)");
}

size_t scalar_bytes(int dtype) { return dtype == SSV_F64 ? sizeof(double) : 2 * sizeof(double); }

// The _dev entry points hand their pointers straight to kernels: a host
// pointer there would make the kernels fault, so it is refused up front.
void require_device_ptr(const void* p, const char* what) {
    if (!p) return;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        ssv::fail(SSV_ERR_INVALID_ARG, std::string(what) + ": not a CUDA pointer (the _dev calls take device memory)");
    }
    if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
        ssv::fail(SSV_ERR_INVALID_ARG,
                  std::string(what) + ": host memory passed to a _dev call (device memory required)");
}

void check_mask(const uint8_t* fd, int n, std::vector<uint8_t>& h, ssv::DevBuf<uint8_t>& d, bool& has) {
    has = fd != nullptr;
    h.clear();
    d.release();
    if (!fd) return;
    h.assign(fd, fd + n);
    for (auto& v : h) v = v ? 1 : 0;
    d.upload(h.data(), h.size(), ssv::stream());
}

// Staging buffer for host-pointer calls.
struct Stage {
    ssv::DevBuf<double> a, b;
    ssv::DevBuf<uint8_t> fd;  // FreeDofs mask of the host-pointer solves (kept: stable address)
};
Stage& stage() {
    static Stage s;
    return s;
}

}  // namespace

extern "C" {

void ssv_version(int* major, int* minor, int* patch) {
    if (major) *major = SSV_VERSION_MAJOR;
    if (minor) *minor = SSV_VERSION_MINOR;
    if (patch) *patch = SSV_VERSION_PATCH;
}

const char* ssv_last_error(void) { return g_last_error.c_str(); }

void ssv_set_loop_guard(int32_t max_loops) { ssv::set_loop_guard(max_loops); }

void ssv_set_alloc_budget(int64_t bytes) { ssv::alloc_budget().store(bytes < 0 ? -1 : (long long)bytes); }

int ssv_device_info(int* count, char* name, int name_cap) {
    return guarded([&] {
        int c = 0;
        if (cudaGetDeviceCount(&c) != cudaSuccess) c = 0;
        if (count) *count = c;
        if (name && name_cap > 0) {
            name[0] = 0;
            if (c > 0) {
                cudaDeviceProp p;
                SSV_CUDA(cudaGetDeviceProperties(&p, 0));
                std::strncpy(name, p.name, name_cap - 1);
                name[name_cap - 1] = 0;
            }
        }
    });
}

void ssv_config_default(ssv_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->tolerance = 1e-10;
    c->max_iterations = 1000;
    c->abs_tolerance = 1e-12;
    c->norm_type = SSV_NORM_RHS;
    c->custom_norm = 1.0;
    c->shift_parameter = 1.05;
    c->shift_increment = 0.05;
    c->max_shift_value = 5.0;
    c->min_diagonal_threshold = 1e-6;
    c->zero_diagonal_replacement = 1e-10;
    c->max_shift_trials = 100;
    c->divergence_threshold = 1000.0;
    c->divergence_count = 100;
    c->save_best_result = 1;
    c->abmc_block_size = 4;
    c->abmc_num_colors = 4;
    c->precision = SSV_PREC_FP64;
}

int ssv_matrix_create(int32_t rows, int32_t cols, const int32_t* row_ptr, const int32_t* col_idx,
                      const void* values, int32_t dtype, ssv_matrix** out) {
    return guarded([&] {
        if (!out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: out is NULL");
        *out = nullptr;
        if (rows < 0 || cols < 0) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: negative size");
        if (dtype != SSV_F64 && dtype != SSV_C128) ssv::fail(SSV_ERR_TYPE, "ssv_matrix_create: unknown dtype");
        if (!row_ptr || (!col_idx && row_ptr[rows] > 0) || (!values && row_ptr[rows] > 0))
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: NULL array");
        if (row_ptr[0] != 0) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: row_ptr[0] must be 0");
        const int64_t nnz = row_ptr[rows];
        for (int i = 0; i < rows; ++i) {
            if (row_ptr[i + 1] < row_ptr[i]) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: row_ptr not monotone");
            for (int k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
                if (col_idx[k] < 0 || col_idx[k] >= cols)
                    ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: column index out of range in row " +
                                                       std::to_string(i));
                if (k > row_ptr[i] && col_idx[k] <= col_idx[k - 1])
                    ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_create: columns of row " + std::to_string(i) +
                                                       " are not sorted and unique");
            }
        }
        require_device();
        auto* A = new ssv_matrix();
        try {
            cudaStream_t s = ssv::stream();
            A->rows = rows;
            A->cols = cols;
            A->nnz = nnz;
            A->dtype = dtype;
            A->h_rp.assign(row_ptr, row_ptr + rows + 1);
            A->h_ci.assign(col_idx, col_idx + nnz);
            A->rp.upload(A->h_rp.data(), A->h_rp.size(), s);
            A->ci.upload(A->h_ci.data(), A->h_ci.size(), s);
            const size_t words = (size_t)nnz * (dtype == SSV_F64 ? 1 : 2);
            A->val.upload(static_cast<const double*>(values), words, s);
            A->lanes = ssv::pick_shape(rows, rows > 0 ? (double)nnz / rows : 1.0);
            SSV_CUDA(cudaStreamSynchronize(s));
        } catch (...) {
            delete A;
            throw;
        }
        *out = A;
    });
}

int ssv_matrix_update_values(ssv_matrix* A, const void* values) {
    return guarded([&] {
        if (!A || !values) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_update_values: NULL argument");
        const size_t words = (size_t)A->nnz * (A->dtype == SSV_F64 ? 1 : 2);
        A->val.alloc(words);
        ssv::h2d_staged(A->val.get(), values, words * sizeof(double), ssv::stream());
        ++A->vgen;
        SSV_CUDA(cudaStreamSynchronize(ssv::stream()));
    });
}

int ssv_matrix_export(const ssv_matrix* A, int32_t* row_ptr, int32_t* col_idx, void* values) {
    return guarded([&] {
        if (!A || !row_ptr || (!col_idx && A->nnz) || (!values && A->nnz))
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_export: NULL argument");
        cudaStream_t s = ssv::stream();
        const size_t words = (size_t)A->nnz * (A->dtype == SSV_F64 ? 1 : 2);
        SSV_CUDA(cudaMemcpyAsync(row_ptr, A->rp.get(), sizeof(int32_t) * (A->rows + 1), cudaMemcpyDeviceToHost, s));
        if (A->nnz) {
            SSV_CUDA(cudaMemcpyAsync(col_idx, A->ci.get(), sizeof(int32_t) * A->nnz, cudaMemcpyDeviceToHost, s));
            SSV_CUDA(cudaMemcpyAsync(values, A->val.get(), sizeof(double) * words, cudaMemcpyDeviceToHost, s));
        }
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_hcurl_assemble(int32_t nv, const double* coords, int32_t nt, const int32_t* tets,
                       const int32_t* tet_edges, const int8_t* signs, int32_t ne,
                       const int32_t* edge_verts, const double* nu, const double* kappa,
                       ssv_matrix** K, ssv_matrix** M, ssv_matrix** G) {
    return guarded([&] {
        if (!K || !M || !G) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: NULL output");
        *K = *M = *G = nullptr;
        if (nv < 0 || nt < 0 || ne < 0) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: negative size");
        if ((nv && !coords) || (nt && (!tets || !tet_edges || !signs)) || (ne && !edge_verts))
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: NULL array");
        for (int64_t q = 0; q < (int64_t)nt * 4; ++q)
            if (tets[q] < 0 || tets[q] >= nv) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: vertex id out of range");
        for (int64_t q = 0; q < (int64_t)nt * 6; ++q) {
            if (tet_edges[q] < 0 || tet_edges[q] >= ne)
                ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: edge id out of range");
            if (signs[q] != 1 && signs[q] != -1) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: signs must be +1 or -1");
        }
        for (int64_t q = 0; q < (int64_t)ne; ++q)
            if (edge_verts[2 * q] < 0 || edge_verts[2 * q] >= edge_verts[2 * q + 1] || edge_verts[2 * q + 1] >= nv)
                ssv::fail(SSV_ERR_INVALID_ARG, "ssv_hcurl_assemble: an edge must list its vertices low, high");
        require_device();
        ssv::hcurl_assemble(nv, coords, nt, tets, tet_edges, signs, ne, edge_verts, nu, kappa, K, M, G);
    });
}

int ssv_matrix_destroy(ssv_matrix* A) {
    return guarded([&] {
        if (!A) return;
        ssv::cocr_forget(A);
        delete A;
    });
}

int ssv_matrix_info(const ssv_matrix* A, int32_t* rows, int32_t* cols, int64_t* nnz, int32_t* dtype) {
    return guarded([&] {
        if (!A) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_info: NULL matrix");
        if (rows) *rows = A->rows;
        if (cols) *cols = A->cols;
        if (nnz) *nnz = A->nnz;
        if (dtype) *dtype = A->dtype;
    });
}

int ssv_matrix_spmv_dev(ssv_matrix* A, const void* d_x, void* d_y) {
    return guarded([&] {
        if (!A || !d_x || !d_y) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_spmv_dev: NULL argument");
        require_device_ptr(d_x, "ssv_matrix_spmv_dev x");
        require_device_ptr(d_y, "ssv_matrix_spmv_dev y");
        ssv::matrix_spmv_dev(A, d_x, d_y);
    });
}

int ssv_matrix_spmv(ssv_matrix* A, const void* x, void* y) {
    return guarded([&] {
        if (!A || !x || !y) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_matrix_spmv: NULL argument");
        cudaStream_t s = ssv::stream();
        const size_t bytes_x = (size_t)A->cols * scalar_bytes(A->dtype);
        const size_t bytes_y = (size_t)A->rows * scalar_bytes(A->dtype);
        Stage& st = stage();
        st.a.alloc(bytes_x / sizeof(double) + 1);
        st.b.alloc(bytes_y / sizeof(double) + 1);
        SSV_CUDA(cudaMemcpyAsync(st.a.get(), x, bytes_x, cudaMemcpyHostToDevice, s));
        ssv::matrix_spmv_dev(A, st.a.get(), st.b.get());
        SSV_CUDA(cudaMemcpyAsync(y, st.b.get(), bytes_y, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_solver_create(ssv_matrix* A, const uint8_t* freedofs, ssv_solver** out) {
    return guarded([&] {
        if (!A || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_solver_create: NULL argument");
        if (A->rows != A->cols) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_solver_create: matrix must be square");
        auto* s = new ssv_solver();
        s->A = A;
        try {
            check_mask(freedofs, A->rows, s->h_fd, s->fd, s->has_fd);
            SSV_CUDA(cudaStreamSynchronize(ssv::stream()));
        } catch (...) {
            delete s;
            throw;
        }
        *out = s;
    });
}

int ssv_solver_destroy(ssv_solver* s) {
    return guarded([&] {
        if (!s) return;
        ssv::mrtr_forget(s);
        delete s;
    });
}

int ssv_solver_solve_dev(ssv_solver* s, const char* method, const ssv_config* cfg, const void* d_b, void* d_x,
                         ssv_result* res, double* history, int32_t history_cap) {
    return guarded([&] {
        if (!s || !cfg || !res || !d_b || !d_x) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_solver_solve_dev: NULL argument");
        require_device_ptr(d_b, "ssv_solver_solve_dev b");
        require_device_ptr(d_x, "ssv_solver_solve_dev x");
        ssv::solver_solve_dev(s, method, *cfg, d_b, d_x, res, history, history_cap);
    });
}

int ssv_solver_solve(ssv_solver* s, const char* method, const ssv_config* cfg, const void* b, void* x,
                     ssv_result* res, double* history, int32_t history_cap) {
    return guarded([&] {
        if (!s || !cfg || !res || !b || !x) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_solver_solve: NULL argument");
        if (ssv::parse_method(method) < 0)
            ssv::fail(SSV_ERR_RUNTIME, std::string("SparseSolvSolver: Unknown method '") + (method ? method : "") +
                                           "'. Available: ICCG, SGSMRTR, CG, COCR");
        cudaStream_t st = ssv::stream();
        const size_t bytes = (size_t)s->A->rows * scalar_bytes(s->A->dtype);
        s->io_b.alloc(bytes / sizeof(double) + 1);
        s->io_x.alloc(bytes / sizeof(double) + 1);
        SSV_CUDA(cudaMemcpyAsync(s->io_b.get(), b, bytes, cudaMemcpyHostToDevice, st));
        SSV_CUDA(cudaMemcpyAsync(s->io_x.get(), x, bytes, cudaMemcpyHostToDevice, st));
        ssv::solver_solve_dev(s, method, *cfg, s->io_b.get(), s->io_x.get(), res, history, history_cap);
        SSV_CUDA(cudaMemcpyAsync(x, s->io_x.get(), bytes, cudaMemcpyDeviceToHost, st));
        SSV_CUDA(cudaStreamSynchronize(st));
    });
}

int ssv_solver_profile(ssv_solver* s, const char* method, const ssv_config* cfg, int32_t reps,
                       ssv_phase_profile* out) {
    return guarded([&] {
        if (!s || !cfg || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_solver_profile: NULL argument");
        ssv::solver_profile(s, method, *cfg, reps, out);
    });
}

int ssv_ic_create(ssv_matrix* A, const uint8_t* freedofs, double shift, ssv_precond** out) {
    return guarded([&] {
        if (!A || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ic_create: NULL argument");
        if (A->rows != A->cols) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ic_create: matrix must be square");
        auto* p = new ssv_precond();
        p->kind = 1;
        p->A = A;
        p->vdtype = A->dtype;
        p->n = A->rows;
        ssv_config_default(&p->cfg);
        p->cfg.shift_parameter = shift;
        try {
            check_mask(freedofs, A->rows, p->h_fd, p->fd, p->has_fd);
            SSV_CUDA(cudaStreamSynchronize(ssv::stream()));
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

int ssv_sgs_create(ssv_matrix* A, const uint8_t* freedofs, ssv_precond** out) {
    return guarded([&] {
        if (!A || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_sgs_create: NULL argument");
        if (A->rows != A->cols) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_sgs_create: matrix must be square");
        auto* p = new ssv_precond();
        p->kind = 4;
        p->A = A;
        p->vdtype = A->dtype;
        p->n = A->rows;
        ssv_config_default(&p->cfg);
        try {
            check_mask(freedofs, A->rows, p->h_fd, p->fd, p->has_fd);
            SSV_CUDA(cudaStreamSynchronize(ssv::stream()));
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

int ssv_amg_create(ssv_matrix* A, const uint8_t* freedofs, double theta, int32_t max_levels, int32_t min_coarse,
                   int32_t num_smooth, ssv_precond** out) {
    return guarded([&] {
        if (!A || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_amg_create: NULL argument");
        if (A->dtype != SSV_F64)
            ssv::fail(SSV_ERR_TYPE, "CompactAMGPreconditioner: expected real SparseMatrix<double>");
        if (A->rows != A->cols) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_amg_create: matrix must be square");
        auto* p = new ssv_precond();
        p->kind = 5;
        p->A = A;
        p->vdtype = SSV_F64;
        p->n = A->rows;
        ssv_config_default(&p->cfg);
        try {
            check_mask(freedofs, A->rows, p->h_fd, p->fd, p->has_fd);
            p->amg.reset(ssv::amg_create(A, p->has_fd ? p->h_fd.data() : nullptr, theta, max_levels, min_coarse,
                                         num_smooth));
            p->ready = true;
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

int ssv_amg_levels(const ssv_precond* p, int32_t* sizes, int32_t cap, int32_t* num_levels) {
    return guarded([&] {
        if (!p || !p->amg || !sizes || !num_levels) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_amg_levels: bad argument");
        *num_levels = ssv::amg_levels(p->amg.get(), sizes, cap);
    });
}

int ssv_ams_create(ssv_matrix* A, ssv_matrix* G, const uint8_t* freedofs, const double* coord_x,
                   const double* coord_y, const double* coord_z, int32_t cycle_type, int32_t num_smooth,
                   double theta, double correction_weight, int32_t complex_form, int32_t ndof_complex,
                   ssv_precond** out) {
    return guarded([&] {
        if (!A || !G || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_create: NULL argument");
        if (A->dtype != SSV_F64 || G->dtype != SSV_F64)
            ssv::fail(SSV_ERR_TYPE, complex_form ? "ComplexCompactAMSPreconditioner: a_real_mat and grad_mat must be real"
                                                 : "CompactAMSPreconditioner: expected real SparseMatrix<double>");
        if (A->rows != A->cols || G->rows != A->rows)
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_create: grad_mat must have one row per row of the matrix");
        if (!coord_x || !coord_y || !coord_z)  // compact_ams.hpp:71-74
            ssv::fail(SSV_ERR_RUNTIME, "CompactAMS: coordinate size mismatch with H1 DOFs");
        const int nc = complex_form && ndof_complex > 0 ? ndof_complex : A->rows;
        if (nc != A->rows)
            ssv::fail(SSV_ERR_INVALID_ARG, "ComplexCompactAMS: ndof_complex must equal the HCurl dimension");
        auto* p = new ssv_precond();
        p->kind = complex_form ? 3 : 2;
        p->A = A;
        p->vdtype = complex_form ? SSV_C128 : SSV_F64;
        p->n = A->rows;
        try {
            check_mask(freedofs, A->rows, p->h_fd, p->fd, p->has_fd);
            p->ams.reset(ssv::ams_create(A, G, p->has_fd ? p->h_fd.data() : nullptr, coord_x, coord_y, coord_z,
                                         cycle_type, num_smooth, theta, correction_weight, complex_form, nc));
            p->ready = true;
        } catch (...) {
            delete p;
            throw;
        }
        *out = p;
    });
}

int ssv_ams_update(ssv_precond* p, ssv_matrix* new_A) {
    return guarded([&] {
        if (!p || !p->ams) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_update: not an AMS preconditioner");
        if (new_A) {  // compact_ams.hpp:89-96
            if (new_A->rows != p->A->rows || new_A->cols != p->A->cols)
                ssv::fail(SSV_ERR_INVALID_ARG, "CompactAMS::Update: new matrix dimension (" +
                                                   std::to_string(new_A->rows) + "x" + std::to_string(new_A->cols) +
                                                   ") does not match original (" + std::to_string(p->A->rows) +
                                                   "x" + std::to_string(p->A->cols) + ")");
            if (new_A->dtype != SSV_F64) ssv::fail(SSV_ERR_TYPE, "CompactAMS::Update: expected a real matrix");
            p->A = new_A;
        }
        p->ready = false;  // an update that fails part way leaves nothing to apply until one succeeds
        ssv::ams_update(p->ams.get(), p->A);
        p->ready = true;
    });
}

int ssv_ams_levels(const ssv_precond* p, int32_t subspace, int32_t* sizes, int32_t cap, int32_t* num_levels) {
    return guarded([&] {
        if (!p || !p->ams || !sizes || !num_levels || subspace < 0 || subspace > 3)
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_levels: bad argument");
        *num_levels = ssv::ams_levels(p->ams.get(), subspace, sizes, cap);
    });
}

int ssv_ams_set_precision(ssv_precond* p, int32_t precision) {
    return guarded([&] {
        if (!p || !p->ams) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_set_precision: not an AMS preconditioner");
        if (precision != SSV_PREC_FP64 && precision != SSV_PREC_FP32 && precision != SSV_PREC_FP32_NODAL)
            ssv::fail(SSV_ERR_INVALID_ARG,
                      "ssv_ams_set_precision: precision must be SSV_PREC_FP64, SSV_PREC_FP32 or SSV_PREC_FP32_NODAL");
        ssv::ams_set_precision(p->ams.get(), precision);
    });
}

int ssv_ams_level_matrix(const ssv_precond* p, int32_t subspace, int32_t level, int32_t what, int32_t* row_ptr,
                         int32_t* col_idx, double* values, int32_t cap, int32_t* nnz, int32_t* on_device) {
    return guarded([&] {
        if (!p || !p->ams || !nnz) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_level_matrix: bad argument");
        *nnz = ssv::ams_level_matrix(p->ams.get(), subspace, level, what, row_ptr, col_idx, values, cap);
        if (on_device) *on_device = ssv::ams_on_device(p->ams.get()) ? 1 : 0;
    });
}

int ssv_ams_subspace_apply(ssv_precond* p, int32_t subspace, const double* r, double* b_s, double* x_s,
                           double* corr) {
    return guarded([&] {
        if (!p || !p->ams || !r || !b_s || !x_s || !corr)
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_subspace_apply: bad argument");
        if (!p->ready) ssv::fail(SSV_ERR_RUNTIME, "CompactAMS::Mult called before Setup");
        ssv::ams_subspace_apply(p->ams.get(), subspace, r, b_s, x_s, corr);
    });
}

int ssv_ams_profile_levels(ssv_precond* p, int32_t subspace, int32_t reps, double* ms_r, double* ms_u,
                           int32_t* shape_r, int32_t* shape_u, int32_t cap, double* last_ms, int32_t* levels) {
    return guarded([&] {
        if (!p || !p->ams || !ms_r || !ms_u || !shape_r || !shape_u || !last_ms || !levels || cap < 0)
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_profile_levels: bad argument");
        if (!p->ready) ssv::fail(SSV_ERR_RUNTIME, "CompactAMS::Mult called before Setup");
        *levels = ssv::ams_profile_levels(p->ams.get(), subspace, reps, ms_r, ms_u, shape_r, shape_u, cap, last_ms);
    });
}

int ssv_ams_setup_times(const ssv_precond* p, double* times) {
    return guarded([&] {
        if (!p || !p->ams || !times) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_setup_times: bad argument");
        ssv::ams_setup_times(p->ams.get(), times);
    });
}

int ssv_ams_profile(ssv_precond* p, int32_t nrhs, int32_t reps, int32_t flags, ssv_phase_profile* out) {
    return guarded([&] {
        if (!p || !p->ams || !out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_profile: bad argument");
        ssv::ams_profile(p->ams.get(), nrhs, reps, flags, out);
    });
}

int ssv_ams_get_precision(const ssv_precond* p, int32_t* precision) {
    return guarded([&] {
        if (!p || !p->ams || !precision) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ams_get_precision: bad argument");
        *precision = ssv::ams_precision(p->ams.get());
    });
}

int ssv_batch_create(ssv_matrix* K, ssv_matrix* M, int32_t num_freq, const double* omegas,
                     ssv_precond* const* pre, int32_t nrhs, const uint8_t* freedofs, ssv_batch** out) {
    return guarded([&] {
        if (!out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_create: NULL out");
        *out = ssv::batch_create(K, M, num_freq, omegas, pre, nrhs, freedofs);
    });
}

int ssv_batch_destroy(ssv_batch* b) {
    return guarded([&] { ssv::batch_destroy(b); });
}

int ssv_batch_cocr_solve(ssv_batch* b, int32_t maxiter, double tol, const void* rhs, void* sol,
                         int32_t* iterations, int32_t* converged, double* residuals) {
    return guarded([&] {
        if (!b || !rhs || !sol) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_cocr_solve: NULL argument");
        ssv::batch_cocr_solve_host(b, maxiter, tol, rhs, sol, iterations, converged, residuals);
    });
}

int ssv_batch_cocr_solve_dev(ssv_batch* b, int32_t maxiter, double tol, const void* d_rhs, void* d_sol,
                             int32_t* iterations, int32_t* converged, double* residuals) {
    return guarded([&] {
        if (!b || !d_rhs || !d_sol) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_cocr_solve_dev: NULL argument");
        require_device_ptr(d_rhs, "ssv_batch_cocr_solve_dev rhs");
        require_device_ptr(d_sol, "ssv_batch_cocr_solve_dev sol");
        ssv::batch_cocr_solve_dev(b, maxiter, tol, d_rhs, d_sol, iterations, converged, residuals);
    });
}

int ssv_batch_tuning(const ssv_batch* b, ssv_batch_tune_entry* entries, int32_t cap, int32_t* count,
                     int32_t* chosen) {
    return guarded([&] {
        if (!b || !count || !chosen || (cap > 0 && !entries))
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_tuning: bad argument");
        int ch = -1;
        *count = ssv::batch_tuning(b, entries, cap, &ch);
        *chosen = ch;
    });
}

int ssv_batch_set_replacement(ssv_batch* b, int32_t every) {
    return guarded([&] {
        if (!b) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_set_replacement: NULL batch");
        ssv::batch_set_replacement(b, every);
    });
}

int ssv_batch_set_refinement(ssv_batch* b, double restart_drop) {
    return guarded([&] {
        if (!b) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_set_refinement: NULL batch");
        ssv::batch_set_refinement(b, restart_drop);
    });
}

int ssv_batch_last_timing(const ssv_batch* b, double* device_ms, double* loop_ms, int32_t* loops,
                          int64_t* kernel_launches) {
    return guarded([&] {
        if (!b) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_last_timing: NULL batch");
        int lp = 0;
        ssv::batch_last_timing(b, device_ms, loop_ms, &lp, kernel_launches, nullptr);
        if (loops) *loops = lp;
    });
}

int ssv_batch_last_cycles(const ssv_batch* b, int32_t* cycles) {
    return guarded([&] {
        if (!b || !cycles) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_batch_last_cycles: NULL argument");
        int c = 0;
        ssv::batch_last_timing(b, nullptr, nullptr, nullptr, nullptr, &c);
        *cycles = c;
    });
}

int ssv_mlp_create(int32_t in_dim, int32_t hidden, uint64_t seed, ssv_mlp** out) {
    return guarded([&] {
        if (!out) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_create: NULL out");
        require_device();
        *out = ssv::mlp_create(in_dim, hidden, seed);
    });
}

int ssv_mlp_destroy(ssv_mlp* m) {
    return guarded([&] { ssv::mlp_destroy(m); });
}

int ssv_mlp_num_params(const ssv_mlp* m, int32_t* count) {
    return guarded([&] {
        if (!m || !count) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_num_params: NULL argument");
        *count = ssv::mlp_nparams(m);
    });
}

int ssv_mlp_get_params(const ssv_mlp* m, float* params) {
    return guarded([&] {
        if (!m || !params) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_get_params: NULL argument");
        ssv::mlp_get_params(m, params);
    });
}

int ssv_mlp_set_params(ssv_mlp* m, const float* params) {
    return guarded([&] {
        if (!m || !params) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_set_params: NULL argument");
        ssv::mlp_set_params(m, params);
    });
}

int ssv_mlp_gradients(ssv_mlp* m, const float* X, const float* y, int64_t n, float* grad, float* loss) {
    return guarded([&] {
        if (!m || !X || !y || !grad || n <= 0) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_gradients: bad argument");
        ssv::mlp_gradients_host(m, X, y, n, grad, loss);
    });
}

int ssv_mlp_train_dev(ssv_mlp* m, const float* d_X, const float* d_y, int64_t n, int32_t epochs, int32_t batch,
                      float lr, uint64_t seed, float* loss) {
    return guarded([&] {
        if (!m || !d_X || !d_y) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_train_dev: NULL argument");
        require_device_ptr(d_X, "ssv_mlp_train_dev X");
        require_device_ptr(d_y, "ssv_mlp_train_dev y");
        ssv::mlp_train_dev(m, d_X, d_y, n, epochs, batch, lr, seed, loss);
    });
}

int ssv_mlp_predict_dev(ssv_mlp* m, const float* d_X, int64_t n, float* d_out) {
    return guarded([&] {
        if (!m || !d_X || !d_out || n < 0) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_mlp_predict_dev: bad argument");
        require_device_ptr(d_X, "ssv_mlp_predict_dev X");
        require_device_ptr(d_out, "ssv_mlp_predict_dev out");
        ssv::mlp_predict_dev(m, d_X, n, d_out);
    });
}

int ssv_pcg_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, const ssv_config* cfg,
                      const void* d_b, void* d_x, ssv_result* res, double* history, int32_t history_cap) {
    return guarded([&] {
        if (!A || !cfg || !res || !d_b || !d_x) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_pcg_solve_dev: NULL argument");
        require_device_ptr(d_b, "ssv_pcg_solve_dev b");
        require_device_ptr(d_x, "ssv_pcg_solve_dev x");
        require_device_ptr(freedofs, "ssv_pcg_solve_dev freedofs");
        ssv::pcg_solve_dev(A, pre, freedofs, *cfg, d_b, d_x, res, history, history_cap);
    });
}

int ssv_pcg_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, const ssv_config* cfg, const void* b,
                  void* x, ssv_result* res, double* history, int32_t history_cap) {
    return guarded([&] {
        if (!A || !cfg || !res || !b || !x) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_pcg_solve: NULL argument");
        cudaStream_t s = ssv::stream();
        const int n = A->rows;
        const size_t bytes = (size_t)n * scalar_bytes(A->dtype);
        Stage& st = stage();
        st.a.alloc(bytes / sizeof(double) + 1);
        st.b.alloc(bytes / sizeof(double) + 1);
        const uint8_t* dfd = nullptr;
        if (freedofs) {
            std::vector<uint8_t> h(freedofs, freedofs + n);
            for (auto& v : h) v = v ? 1 : 0;
            st.fd.upload(h.data(), h.size(), s);
            dfd = st.fd.get();
        }
        SSV_CUDA(cudaMemcpyAsync(st.a.get(), b, bytes, cudaMemcpyHostToDevice, s));
        SSV_CUDA(cudaMemcpyAsync(st.b.get(), x, bytes, cudaMemcpyHostToDevice, s));
        ssv::pcg_solve_dev(A, pre, dfd, *cfg, st.a.get(), st.b.get(), res, history, history_cap);
        SSV_CUDA(cudaMemcpyAsync(x, st.b.get(), bytes, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_ic_set_config(ssv_precond* p, const ssv_config* cfg) {
    return guarded([&] {
        if (!p || !cfg) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ic_set_config: NULL argument");
        p->cfg = *cfg;
    });
}

int ssv_precond_update(ssv_precond* p) {
    return guarded([&] {
        if (!p) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_precond_update: NULL preconditioner");
        p->ready = false;  // an update that fails part way leaves nothing to apply until one succeeds
        if (p->ams) ssv::ams_update(p->ams.get(), p->A);
        else ssv::precond_update(p);
        p->ready = true;
    });
}

int ssv_precond_apply_dev(ssv_precond* p, const void* d_x, void* d_y) {
    return guarded([&] {
        if (!p || !d_x || !d_y) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_precond_apply_dev: NULL argument");
        require_device_ptr(d_x, "ssv_precond_apply_dev x");
        require_device_ptr(d_y, "ssv_precond_apply_dev y");
        ssv::precond_apply_dev(p, d_x, d_y);
    });
}

int ssv_precond_apply(ssv_precond* p, const void* x, void* y) {
    return guarded([&] {
        if (!p || !x || !y) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_precond_apply: NULL argument");
        if (!p->ready) ssv::fail(SSV_ERR_RUNTIME, "ICPreconditioner::apply called before setup");
        cudaStream_t s = ssv::stream();
        const size_t bytes = (size_t)p->n * scalar_bytes(p->vdtype);
        p->io_x.alloc(bytes / sizeof(double) + 1);
        p->io_y.alloc(bytes / sizeof(double) + 1);
        SSV_CUDA(cudaMemcpyAsync(p->io_x.get(), x, bytes, cudaMemcpyHostToDevice, s));
        ssv::precond_apply_dev(p, p->io_x.get(), p->io_y.get());
        SSV_CUDA(cudaMemcpyAsync(y, p->io_y.get(), bytes, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_precond_apply_block(ssv_precond* p, int32_t nrhs, const void* x, void* y) {
    return guarded([&] {
        if (!p || !x || !y) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_precond_apply_block: NULL argument");
        if ((p->kind != 2 && p->kind != 3) || !p->ams)
            ssv::fail(SSV_ERR_TYPE, "ssv_precond_apply_block: CompactAMS / ComplexCompactAMS handles only");
        if (nrhs != 1 && nrhs != 4) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_precond_apply_block: nrhs must be 1 or 4");
        if (!p->ready) ssv::fail(SSV_ERR_RUNTIME, "CompactAMS::Mult called before Setup");
        cudaStream_t s = ssv::stream();
        const size_t bytes = (size_t)p->n * nrhs * scalar_bytes(p->vdtype);
        p->io_x.alloc(bytes / sizeof(double) + 1);
        p->io_y.alloc(bytes / sizeof(double) + 1);
        SSV_CUDA(cudaMemcpyAsync(p->io_x.get(), x, bytes, cudaMemcpyHostToDevice, s));
        ssv::ams_reserve_block(p->ams.get(), nrhs);
        ssv::ams_apply_block(p->ams.get(), p->io_x.get(), p->io_y.get(), nrhs, nullptr, s);
        SSV_CUDA(cudaMemcpyAsync(y, p->io_y.get(), bytes, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_ic_actual_shift(const ssv_precond* p, double* shift) {
    return guarded([&] {
        if (!p || !shift) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_ic_actual_shift: NULL argument");
        *shift = ssv::precond_actual_shift(p);
    });
}

int ssv_precond_destroy(ssv_precond* p) {
    return guarded([&] { delete p; });
}

int ssv_cocr_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                       int32_t printrates, const void* d_b, void* d_x, int32_t* iterations) {
    return guarded([&] {
        if (!A || !d_b || !d_x || !iterations) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_cocr_solve_dev: NULL argument");
        require_device_ptr(d_b, "ssv_cocr_solve_dev b");
        require_device_ptr(d_x, "ssv_cocr_solve_dev x");
        require_device_ptr(freedofs, "ssv_cocr_solve_dev freedofs");
        ssv::cocr_solve_dev(A, pre, freedofs, maxiter, tol, printrates, d_b, d_x, iterations);
    });
}

int ssv_cocr_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                   int32_t printrates, const void* b, void* x, int32_t* iterations) {
    return guarded([&] {
        if (!A || !b || !x || !iterations) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_cocr_solve: NULL argument");
        cudaStream_t s = ssv::stream();
        const int n = A->rows;
        const size_t bytes = (size_t)n * scalar_bytes(A->dtype);
        Stage& st = stage();
        st.a.alloc(bytes / sizeof(double) + 1);
        st.b.alloc(bytes / sizeof(double) + 1);
        const uint8_t* dfd = nullptr;
        if (freedofs) {
            std::vector<uint8_t> h(freedofs, freedofs + n);
            for (auto& v : h) v = v ? 1 : 0;
            st.fd.upload(h.data(), h.size(), s);
            dfd = st.fd.get();
        }
        SSV_CUDA(cudaMemcpyAsync(st.a.get(), b, bytes, cudaMemcpyHostToDevice, s));
        ssv::cocr_solve_dev(A, pre, dfd, maxiter, tol, printrates, st.a.get(), st.b.get(), iterations);
        SSV_CUDA(cudaMemcpyAsync(x, st.b.get(), bytes, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_cocr_last_launches(int64_t* launches) {
    return guarded([&] {
        if (!launches) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_cocr_last_launches: NULL argument");
        *launches = ssv::cocr_last_launches();
    });
}

int ssv_cocr_refined_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter,
                               double tol, double restart_drop, int32_t printrates, const void* d_b,
                               void* d_x, ssv_refine_info* info) {
    return guarded([&] {
        if (!A || !d_b || !d_x) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_cocr_refined_solve_dev: NULL argument");
        require_device_ptr(d_b, "ssv_cocr_refined_solve_dev b");
        require_device_ptr(d_x, "ssv_cocr_refined_solve_dev x");
        require_device_ptr(freedofs, "ssv_cocr_refined_solve_dev freedofs");
        ssv::cocr_refined_solve_dev(A, pre, freedofs, maxiter, tol, restart_drop, printrates, d_b, d_x, info);
    });
}

int ssv_cocr_refined_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                           double restart_drop, int32_t printrates, const void* b, void* x,
                           ssv_refine_info* info) {
    return guarded([&] {
        if (!A || !b || !x) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_cocr_refined_solve: NULL argument");
        cudaStream_t s = ssv::stream();
        const int n = A->rows;
        const size_t bytes = (size_t)n * scalar_bytes(A->dtype);
        Stage& st = stage();
        st.a.alloc(bytes / sizeof(double) + 1);
        st.b.alloc(bytes / sizeof(double) + 1);
        const uint8_t* dfd = nullptr;
        if (freedofs) {
            std::vector<uint8_t> h(freedofs, freedofs + n);
            for (auto& v : h) v = v ? 1 : 0;
            st.fd.upload(h.data(), h.size(), s);
            dfd = st.fd.get();
        }
        SSV_CUDA(cudaMemcpyAsync(st.a.get(), b, bytes, cudaMemcpyHostToDevice, s));
        ssv::cocr_refined_solve_dev(A, pre, dfd, maxiter, tol, restart_drop, printrates, st.a.get(), st.b.get(),
                                    info);
        SSV_CUDA(cudaMemcpyAsync(x, st.b.get(), bytes, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_gmres_solve_dev(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                        int32_t restart, const void* d_b, void* d_x, int32_t* iterations) {
    return guarded([&] {
        if (!A || !d_b || !d_x || !iterations) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_gmres_solve_dev: NULL argument");
        if (A->rows != A->cols) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_gmres_solve_dev: matrix must be square");
        require_device_ptr(d_b, "ssv_gmres_solve_dev b");
        require_device_ptr(d_x, "ssv_gmres_solve_dev x");
        require_device_ptr(freedofs, "ssv_gmres_solve_dev freedofs");
        ssv::gmres_solve_dev(A, pre, freedofs, maxiter, tol, restart, d_b, d_x, iterations);
    });
}

int ssv_gmres_solve(ssv_matrix* A, ssv_precond* pre, const uint8_t* freedofs, int32_t maxiter, double tol,
                    int32_t restart, const void* b, void* x, int32_t* iterations) {
    return guarded([&] {
        if (!A || !b || !x || !iterations) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_gmres_solve: NULL argument");
        if (A->rows != A->cols) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_gmres_solve: matrix must be square");
        cudaStream_t s = ssv::stream();
        const int n = A->rows;
        const size_t bytes = (size_t)n * scalar_bytes(A->dtype);
        Stage& st = stage();
        st.a.alloc(bytes / sizeof(double) + 1);
        st.b.alloc(bytes / sizeof(double) + 1);
        const uint8_t* dfd = nullptr;
        if (freedofs) {
            std::vector<uint8_t> h(freedofs, freedofs + n);
            for (auto& v : h) v = v ? 1 : 0;
            st.fd.upload(h.data(), h.size(), s);
            dfd = st.fd.get();
        }
        SSV_CUDA(cudaMemcpyAsync(st.a.get(), b, bytes, cudaMemcpyHostToDevice, s));
        ssv::gmres_solve_dev(A, pre, dfd, maxiter, tol, restart, st.a.get(), st.b.get(), iterations);
        SSV_CUDA(cudaMemcpyAsync(x, st.b.get(), bytes, cudaMemcpyDeviceToHost, s));
        SSV_CUDA(cudaStreamSynchronize(s));
    });
}

int ssv_abmc_build(int32_t n, const int32_t* row_ptr, const int32_t* col_idx, int32_t block_size,
                   int32_t target_colors, int32_t* num_colors, int32_t* num_blocks, int32_t* color_offsets,
                   int32_t* block_offsets, int32_t* ordering, int32_t* reverse_ordering) {
    return guarded([&] {
        if (n < 0 || (n > 0 && (!row_ptr || !col_idx))) ssv::fail(SSV_ERR_INVALID_ARG, "ssv_abmc_build: bad input");
        ssv::AbmcSchedule s;
        ssv::build_abmc(n, row_ptr, col_idx, block_size, target_colors, s);
        *num_colors = s.num_colors;
        *num_blocks = s.num_blocks;
        if (n <= 0) return;
        std::memcpy(color_offsets, s.color_offsets.data(), sizeof(int) * s.color_offsets.size());
        std::memcpy(block_offsets, s.block_offsets.data(), sizeof(int) * s.block_offsets.size());
        std::memcpy(ordering, s.ordering.data(), sizeof(int) * n);
        std::memcpy(reverse_ordering, s.reverse.data(), sizeof(int) * n);
    });
}

int ssv_level_schedule(int32_t n, const int32_t* row_ptr, const int32_t* col_idx, int32_t upper,
                       int32_t* level_of, int32_t* num_levels) {
    return guarded([&] {
        std::vector<int> lev;
        *num_levels = ssv::build_levels(n, row_ptr, col_idx, upper != 0, lev);
        if (n > 0) std::memcpy(level_of, lev.data(), sizeof(int) * n);
    });
}

int ssv_rcm_order(int32_t n, const int32_t* row_ptr, const int32_t* col_idx, int32_t* ordering,
                  int32_t* reverse_ordering) {
    return guarded([&] {
        if (n < 0 || (n > 0 && (!row_ptr || !col_idx || !ordering || !reverse_ordering)))
            ssv::fail(SSV_ERR_INVALID_ARG, "ssv_rcm_order: bad input");
        std::vector<int> o, r;
        ssv::rcm_order(n, row_ptr, col_idx, o, r);
        if (n <= 0) return;
        std::memcpy(ordering, o.data(), sizeof(int) * n);
        std::memcpy(reverse_ordering, r.data(), sizeof(int) * n);
    });
}

}  // extern "C"

// Error text for ssv_spmv_dot_noalloc (noalloc.cu), which reports through the
// same thread-local message as every other entry point.
namespace ssv {
const char* noalloc_set_error(const std::string& m) {
    g_last_error = m;
    return g_last_error.c_str();
}
}  // namespace ssv
