// Host runtime and the C ABI of include/owtk.h: context, device vectors,
// matrices, preconditioners (including the ILU symbolic phase) and the
// entry points.  Solver recurrences live in solvers.cpp.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <string>
#include <utility>

#include <cuda_bf16.h>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {

namespace {
thread_local std::string g_last_error;
}

void fail(owtk_status code, const std::string& message) { throw Error{code, message}; }

void record_error(const std::string& message) { g_last_error = message; }

void cuda_check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess) fail(OWTK_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

DeviceBuffer& DeviceBuffer::operator=(DeviceBuffer&& o) noexcept
{
    if (this != &o) {
        if (ptr) cudaFree(ptr);
        ptr = o.ptr;
        bytes = o.bytes;
        o.ptr = nullptr;
        o.bytes = 0;
    }
    return *this;
}

DeviceBuffer::~DeviceBuffer()
{
    if (ptr) cudaFree(ptr);
}

void DeviceBuffer::allocate(std::size_t n)
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = n;
    if (n) OWTK_CUDA(cudaMalloc(&ptr, n));
}

Context::~Context()
{
    if (stream) cudaStreamSynchronize(stream);
    if (host_scalars) cudaFreeHost(host_scalars);
    if (stream) cudaStreamDestroy(stream);
}

void Context::sync() { OWTK_CUDA(cudaStreamSynchronize(stream)); }

void Context::check_device_status()
{
    unsigned word = 0;
    OWTK_CUDA(cudaMemcpyAsync(&word, status.ptr, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    sync();
    if (word == 0) return;
    OWTK_CUDA(cudaMemsetAsync(status.ptr, 0, sizeof(unsigned), stream));
    sync();
    if (word & dev::kErrTimeout)
        fail(OWTK_ERR_TIMEOUT, "a device sweep gave up waiting for a dependency");
    if (word & dev::kErrZeroPivot) fail(OWTK_ERR_ZERO_PIVOT, "zero pivot in ILU(0)");
    if (word & dev::kErrMissingDiagonal) fail(OWTK_ERR_INVALID_ARGUMENT, "row has no diagonal");
    if (word & dev::kErrSingularDiagonal) fail(OWTK_ERR_INVALID_ARGUMENT, "singular diagonal");
}

void Workspace::prepare(const Vector& layout, std::size_t count, std::size_t scalars)
{
    const bool changed = vectors.empty() || !vectors.front()->same_layout(layout)
        || vectors.front()->dtype != layout.dtype;
    if (changed || vectors.size() < count) {
        vectors.clear();
        for (std::size_t i = 0; i < count; ++i) {
            auto v = std::make_unique<owtk_vector>();
            v->ctx = ctx;
            v->dtype = layout.dtype;
            v->owned = layout.owned;
            v->ghost = layout.ghost;
            v->bs = layout.bs;
            v->storage.allocate(layout.local_size() * layout.elem());
            OWTK_CUDA(cudaMemsetAsync(v->storage.ptr, 0, layout.local_size() * layout.elem(), ctx->stream));
            v->data = v->storage.ptr;
            vectors.push_back(std::move(v));
        }
        ++epochs;
    }
    if (scalar_capacity < scalars) {
        scalar_capacity = scalars;
        ++epochs;
    }
}

// ------------------------------------------------------------ helpers
namespace {

std::size_t dsize(owtk_dtype d) { return d == OWTK_F64 ? 8 : (d == OWTK_F32 ? 4 : 2); }

// Validate a host CSR structure as block_csr.hpp:281-300 does and narrow it
// to int32 for the device.
void ingest_structure(Matrix& m, std::size_t owned, std::size_t ghost, std::size_t bs,
                      const std::uint64_t* rowptr, const std::uint64_t* cols, const char* what)
{
    require(rowptr != nullptr && cols != nullptr, what);
    require(owned != 0 && bs != 0 && rowptr[0] == 0, what);
    const std::uint64_t nnz = rowptr[owned];
    require(owned + ghost < static_cast<std::size_t>(std::numeric_limits<std::int32_t>::max())
                && nnz < static_cast<std::uint64_t>(std::numeric_limits<std::int32_t>::max()),
            "matrix too large for 32-bit device indices");
    m.owned = owned;
    m.ghost = ghost;
    m.bs = bs;
    m.entries = nnz;
    m.h_rowptr.resize(owned + 1);
    for (std::size_t r = 0; r <= owned; ++r) {
        if (r < owned && rowptr[r] > rowptr[r + 1])
            fail(OWTK_ERR_INVALID_ARGUMENT, "nonmonotone BlockCsrMatrix offsets");
        m.h_rowptr[r] = static_cast<std::int32_t>(rowptr[r]);
    }
    m.h_cols.resize(nnz);
    for (std::uint64_t e = 0; e < nnz; ++e) {
        if (cols[e] >= owned + ghost)
            fail(OWTK_ERR_INVALID_ARGUMENT, "BlockCsrMatrix column outside local layout");
        m.h_cols[e] = static_cast<std::int32_t>(cols[e]);
    }
    m.rowptr = upload(m.ctx->stream, m.h_rowptr);
    m.cols = upload(m.ctx->stream, m.h_cols);
    build_tile_plan(m);
}

template<class T> void matrix_layout_check(const Matrix& m, const Vector& in, const Vector& out)
{
    if (!in.same_layout(out) || in.owned != m.owned || in.ghost != m.ghost || in.bs != m.bs)
        fail(OWTK_ERR_INVALID_ARGUMENT, "BlockCsrMatrix vector layout mismatch");
    if (in.dtype != m.dtype || out.dtype != m.dtype)
        fail(OWTK_ERR_INVALID_ARGUMENT, "vector dtype differs from matrix dtype");
}

// -------------------------------------------------------------- ILU symbolic
// preconditioner.hpp:373-427: ghost columns dropped, columns sorted,
// level(i,j) = min(level(i,p) + level(p,j) + 1) kept while <= k; duplicate
// columns and missing diagonals are rejected.
void ilu_symbolic(Preconditioner& p, const Matrix& m, std::size_t fill)
{
    const std::size_t n = m.owned;
    p.f_rowptr.assign(1, 0);
    p.f_cols.clear();
    p.f_source.clear();
    p.f_diagpos.assign(n, 0);
    p.row_counts.assign(n, 0);
    std::vector<std::int32_t> levels;
    struct Item { std::int32_t col; std::size_t level; std::int64_t source; };
    std::vector<Item> row;
    for (std::size_t r = 0; r < n; ++r) {
        row.clear();
        for (std::int32_t s = m.h_rowptr[r]; s < m.h_rowptr[r + 1]; ++s) {
            const std::int32_t c = m.h_cols[s];
            if (static_cast<std::size_t>(c) >= n) continue;
            row.push_back({c, 0, s});
            ++p.row_counts[r];
        }
        std::sort(row.begin(), row.end(), [](const Item& a, const Item& b) { return a.col < b.col; });
        for (std::size_t i = 1; i < row.size(); ++i)
            if (row[i].col == row[i - 1].col)
                fail(OWTK_ERR_INVALID_ARGUMENT, "ILU requires unique matrix columns");
        if (fill > 0) {
            // Visit pivots in column order; fill inserted to the right of the
            // current pivot is visited later (std::map iteration order).
            for (std::size_t k = 0; k < row.size() && static_cast<std::size_t>(row[k].col) < r; ++k) {
                const std::int32_t pivot = row[k].col;
                const std::size_t lower = row[k].level;
                if (lower >= fill) continue;
                for (std::int32_t u = p.f_diagpos[pivot] + 1; u < p.f_rowptr[pivot + 1]; ++u) {
                    const auto ul = static_cast<std::size_t>(levels[u]);
                    if (ul > fill - lower - 1) continue;
                    const std::size_t level = lower + ul + 1;
                    const std::int32_t col = p.f_cols[u];
                    auto it = std::lower_bound(row.begin(), row.end(), col,
                                               [](const Item& a, std::int32_t c) { return a.col < c; });
                    if (it != row.end() && it->col == col) it->level = std::min(it->level, level);
                    else row.insert(it, {col, level, -1});
                }
            }
        }
        bool found = false;
        for (const Item& it : row) {
            if (static_cast<std::size_t>(it.col) == r) {
                p.f_diagpos[r] = static_cast<std::int32_t>(p.f_cols.size());
                found = true;
            }
            p.f_cols.push_back(it.col);
            levels.push_back(static_cast<std::int32_t>(it.level));
            p.f_source.push_back(it.source);
        }
        if (!found) fail(OWTK_ERR_INVALID_ARGUMENT, "ILU(0) row has no diagonal");
        p.f_rowptr.push_back(static_cast<std::int32_t>(p.f_cols.size()));
    }
    // IKJ update lists (preconditioner.hpp:456-468): for lower entry l of row
    // r with pivot row q, the (target, upper) pairs in upper order, skipping
    // columns absent from row r.
    const std::size_t nnz = p.f_cols.size();
    std::vector<std::int32_t> start(nnz + 1, 0), target, upper;
    std::vector<std::int32_t> pos(n, -1);
    for (std::size_t r = 0; r < n; ++r) {
        for (std::int32_t e = p.f_rowptr[r]; e < p.f_rowptr[r + 1]; ++e) pos[p.f_cols[e]] = e;
        for (std::int32_t e = p.f_rowptr[r]; e < p.f_rowptr[r + 1]; ++e) {
            if (e < p.f_diagpos[r]) {
                const std::int32_t q = p.f_cols[e];
                for (std::int32_t u = p.f_diagpos[q] + 1; u < p.f_rowptr[q + 1]; ++u) {
                    const std::int32_t t = pos[p.f_cols[u]];
                    if (t < 0) continue;
                    target.push_back(t);
                    upper.push_back(u);
                }
            }
            start[static_cast<std::size_t>(e) + 1] = static_cast<std::int32_t>(target.size());
        }
        for (std::int32_t e = p.f_rowptr[r]; e < p.f_rowptr[r + 1]; ++e) pos[p.f_cols[e]] = -1;
    }
    cudaStream_t s = p.ctx->stream;
    p.d_frowptr = upload(s, p.f_rowptr);
    p.d_fcols = upload(s, p.f_cols);
    p.d_fdiagpos = upload(s, p.f_diagpos);
    p.d_fsource = upload(s, p.f_source);
    p.d_upd_start = upload(s, start);
    p.d_upd_target = upload(s, target);
    p.d_upd_upper = upload(s, upper);
    const std::size_t per = p.block ? p.bs * p.bs : p.bs;   // values per factor entry
    p.d_fvalues.allocate(nnz * per * dsize(p.dtype) + 16);
    p.inv_diag.allocate(n * per * dsize(p.dtype) + 16);
    p.work.allocate(n * p.bs * dsize(p.dtype) + 16);   // forward-sweep result of an apply
    std::vector<std::int32_t> lower_level, upper_level;
    levels_of(n, p.f_rowptr.data(), p.f_cols.data(), lower_level, upper_level);
    build_sweep(*p.ctx, p.lower, n, p.bs, lower_level, false);
    build_sweep(*p.ctx, p.upper, n, p.bs, upper_level, true);
    if (!p.block) {
        build_chain_sweep(*p.ctx, p.chain, n, p.lower.depth, p.upper.depth, p.f_rowptr);
    }
    if (!p.block && !p.chain.ready) {
        build_lockstep_sweep(*p.ctx, p.l_lower, n, p.bs, m.dtype, lower_level, p.f_rowptr, p.f_cols, p.f_diagpos,
                             false);
        if (p.l_lower.ready)
            build_lockstep_sweep(*p.ctx, p.l_upper, n, p.bs, m.dtype, upper_level, p.f_rowptr, p.f_cols,
                                 p.f_diagpos, true);
        if (!p.l_lower.ready || !p.l_upper.ready) p.l_lower.ready = p.l_upper.ready = false;
    }
    if (!p.block && !p.chain.ready && !p.l_lower.ready) {
        std::vector<std::uint32_t> loc;
        build_cluster_sweep(*p.ctx, p.c_lower, n, p.bs, m.dtype, lower_level, p.f_rowptr, p.f_cols, p.f_diagpos,
                            false, loc);
        if (p.c_lower.ready)
            build_cluster_sweep(*p.ctx, p.c_upper, n, p.bs, m.dtype, upper_level, p.f_rowptr, p.f_cols,
                                p.f_diagpos, true, loc);
        if (p.c_lower.ready && p.c_upper.ready) p.d_floc = upload(p.ctx->stream, loc);
        else p.c_lower.ready = p.c_upper.ready = false;
    }
}

// preconditioner.hpp:269-311: the new matrix must have the analysed pattern.
void ilu_pattern_check(const Preconditioner& p, const Matrix& m)
{
    if (m.owned != p.owned || m.ghost != p.ghost || m.bs != p.bs)
        fail(OWTK_ERR_INVALID_ARGUMENT, "ILU(0) matrix layout mismatch");
    for (std::size_t r = 0; r < p.owned; ++r) {
        std::int32_t count = 0;
        for (std::int32_t s = m.h_rowptr[r]; s < m.h_rowptr[r + 1]; ++s)
            count += static_cast<std::size_t>(m.h_cols[s]) < p.owned;
        if (count != p.row_counts[r]) fail(OWTK_ERR_INVALID_ARGUMENT, "ILU(0) sparsity pattern changed");
        for (std::int32_t d = p.f_rowptr[r]; d < p.f_rowptr[r + 1]; ++d) {
            const std::int64_t s = p.f_source[d];
            if (s < 0) continue;
            if (s < m.h_rowptr[r] || s >= m.h_rowptr[r + 1] || m.h_cols[s] != p.f_cols[d])
                fail(OWTK_ERR_INVALID_ARGUMENT, "ILU(0) sparsity pattern changed");
        }
    }
}

template<class T> void ilu_numeric(Preconditioner& p, const Matrix& m)
{
    kern::ilu_factorize<T>(*p.ctx, p, static_cast<const T*>(m.values.ptr));
    p.ctx->check_device_status();
}

template<class T> void jacobi_setup(Preconditioner& p, const Matrix& m)
{
    Context& c = *p.ctx;
    const std::size_t n = m.owned * m.bs;
    DeviceBuffer d(n * sizeof(T) + 16);
    const T* diag;
    if (m.kind == 0) {
        kern::bsr_diagonal<T>(c, m, d.as<T>());
        diag = d.as<T>();
        try {
            c.check_device_status();
        } catch (const Error&) {
            fail(OWTK_ERR_INVALID_ARGUMENT, "BlockCsrMatrix row has no diagonal");
        }
    } else {
        diag = static_cast<const T*>(m.diag);
    }
    const T minimum = p.parameter > 0 ? static_cast<T>(p.parameter)
                                      : T(64) * std::numeric_limits<T>::epsilon();
    kern::reciprocal_checked<T>(c, n, diag, minimum, p.inv_diag.as<T>());
    try {
        c.check_device_status();
    } catch (const Error&) {
        fail(OWTK_ERR_INVALID_ARGUMENT, "Jacobi preconditioner has a singular diagonal");
    }
}

template<class T> void ssor_setup(Preconditioner& p, const Matrix& m)
{
    Context& c = *p.ctx;
    const std::size_t n = m.owned * m.bs;
    const T* diag;
    if (p.kind == OWTK_PC_SSOR) {
        kern::bsr_diagonal<T>(c, m, p.diag_cache.as<T>());
        try {
            c.check_device_status();
        } catch (const Error&) {
            fail(OWTK_ERR_INVALID_ARGUMENT, "SSOR preconditioner row has no diagonal");
        }
        diag = p.diag_cache.as<T>();
    } else {
        diag = static_cast<const T*>(m.diag);
    }
    // Singular-diagonal check (preconditioner.hpp:159-163, split_block_csr.hpp:234-239);
    // the reciprocals themselves are scratch.
    kern::reciprocal_checked<T>(c, n, diag, T(64) * std::numeric_limits<T>::epsilon(), p.work.as<T>());
    try {
        c.check_device_status();
    } catch (const Error&) {
        fail(OWTK_ERR_INVALID_ARGUMENT, p.kind == OWTK_PC_SSOR ? "SSOR preconditioner has a singular diagonal"
                                                               : "split SSOR has a singular diagonal");
    }
}

// Low-precision factor copies of an FP64 factorisation.
void store_factors(Preconditioner& p)
{
    if (p.storage == OWTK_F64) return;
    Context& c = *p.ctx;
    const std::size_t per = p.block ? p.bs * p.bs : p.bs;
    const std::size_t nv = p.f_cols.size() * per, ni = p.owned * per;
    if (p.storage == OWTK_F32) {
        kern::convert<float, double>(c, nv, p.d_fvalues.as<double>(), p.lp_vals.as<float>());
        kern::convert<float, double>(c, ni, p.inv_diag.as<double>(), p.lp_inv.as<float>());
    } else {
        kern::convert<__nv_bfloat16, double>(c, nv, p.d_fvalues.as<double>(), p.lp_vals.as<__nv_bfloat16>());
        kern::convert<__nv_bfloat16, double>(c, ni, p.inv_diag.as<double>(), p.lp_inv.as<__nv_bfloat16>());
    }
}

void numeric_update(Preconditioner& p, Matrix& m);

void mixed_update(Preconditioner& p, Matrix& m)
{
    const std::size_t per = m.kind == 2 ? m.bs * m.bs : m.bs;
    kern::convert<float, double>(*p.ctx, m.entries * per, m.values.as<double>(), p.m32->values.as<float>());
    kern::slices_fill(*p.ctx, *p.m32);
    numeric_update(*p.inner, m);
}

void numeric_update(Preconditioner& p, Matrix& m)
{
    if (p.kind == OWTK_PC_MIXED) {
        mixed_update(p, m);
    } else if (p.dtype == OWTK_F64) {
        if (p.kind == OWTK_PC_JACOBI) jacobi_setup<double>(p, m);
        else if (p.kind == OWTK_PC_SSOR || p.kind == OWTK_PC_SPLIT_SSOR) ssor_setup<double>(p, m);
        else if (p.kind == OWTK_PC_ILU) ilu_numeric<double>(p, m);
        else if (p.kind == OWTK_PC_BLOCK_ILU) {
            kern::block_ilu_factorize(*p.ctx, p, m.values.as<double>());
            p.ctx->check_device_status();
        }
        store_factors(p);
    } else {
        if (p.kind == OWTK_PC_JACOBI) jacobi_setup<float>(p, m);
        else if (p.kind == OWTK_PC_SSOR || p.kind == OWTK_PC_SPLIT_SSOR) ssor_setup<float>(p, m);
        else if (p.kind == OWTK_PC_ILU) ilu_numeric<float>(p, m);
    }
    ++p.numeric_updates;
}

}  // namespace

// ------------------------------------------------------------ host callbacks
namespace {
// One application of a host function: in and the current out copied to host
// buffers, the function called, out's owned values and in's ghost values
// (which a halo exchange of the application may write) copied back.
void host_apply_call(Context& c, owtk_host_apply_fn fn, void* user, std::vector<unsigned char>& hin,
                     std::vector<unsigned char>& hout, Vector& in, Vector& out)
{
    const std::size_t count = in.local_size(), es = in.elem(), bytes = count * es;
    hin.resize(bytes);
    hout.resize(bytes);
    OWTK_CUDA(cudaMemcpyAsync(hin.data(), in.data, bytes, cudaMemcpyDeviceToHost, c.stream));
    OWTK_CUDA(cudaMemcpyAsync(hout.data(), out.data, bytes, cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    if (fn(user, hin.data(), hout.data(), count) != 0) fail(OWTK_ERR_RUNTIME, "host apply callback failed");
    const std::size_t owned_bytes = in.owned_size() * es;
    OWTK_CUDA(cudaMemcpyAsync(out.data, hout.data(), owned_bytes, cudaMemcpyHostToDevice, c.stream));
    if (in.ghost > 0 && in.data != out.data)
        OWTK_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(in.data) + owned_bytes, hin.data() + owned_bytes,
                                  bytes - owned_bytes, cudaMemcpyHostToDevice, c.stream));
    c.sync();
}
}  // namespace

std::unique_ptr<Vector> make_vector_like(const Vector& like)
{
    auto v = std::make_unique<owtk_vector>();
    v->ctx = like.ctx;
    v->dtype = like.dtype;
    v->owned = like.owned;
    v->ghost = like.ghost;
    v->bs = like.bs;
    v->storage.allocate(like.local_size() * like.elem() + 16);
    v->data = v->storage.ptr;
    OWTK_CUDA(cudaMemsetAsync(v->data, 0, like.local_size() * like.elem(), like.ctx->stream));
    return v;
}

// ------------------------------------------------------------ Arnoldi snapshot
// core.hpp:462-534.
void ArnoldiSnapshot::begin_cycle(const Vector& layout, std::size_t maximum_columns)
{
    max_columns = maximum_columns;
    columns = 0;
    h.assign((maximum_columns + 1) * maximum_columns, 0.0);
    if (basis.size() < maximum_columns
        || (!basis.empty() && (!basis.front()->same_layout(layout) || basis.front()->dtype != layout.dtype))) {
        basis.clear();
        basis.reserve(maximum_columns);
        for (std::size_t i = 0; i < maximum_columns; ++i) basis.push_back(make_vector_like(layout));
    }
}

void ArnoldiSnapshot::record_column(std::size_t column, const double* values, std::size_t count)
{
    if (column >= max_columns || count != column + 2)
        fail(OWTK_ERR_INVALID_ARGUMENT, "invalid Arnoldi snapshot column");
    for (std::size_t row = 0; row < count; ++row) h[column * (max_columns + 1) + row] = values[row];
}

void ArnoldiSnapshot::finish_cycle(const std::vector<Vector*>& preconditioned, std::size_t count)
{
    if (count > max_columns || preconditioned.size() < count)
        fail(OWTK_ERR_INVALID_ARGUMENT, "invalid Arnoldi snapshot basis");
    columns = count;
    for (std::size_t col = 0; col < count; ++col) {
        const Vector& z = *preconditioned[col];
        OWTK_CUDA(cudaMemcpyAsync(basis[col]->data, z.data, z.owned_size() * z.elem(), cudaMemcpyDeviceToDevice,
                                  z.ctx->stream));
    }
}

void ArnoldiSnapshot::clear()
{
    columns = 0;
    max_columns = 0;
    h.clear();
    basis.clear();
}

// ------------------------------------------------------------ shared ops
void apply_operator(Matrix& m, Vector& in, Vector& out)
{
    if (m.kind == 3) {
        if (!in.same_layout(out) || in.owned != m.owned || in.ghost != m.ghost || in.bs != m.bs)
            fail(OWTK_ERR_INVALID_ARGUMENT, "operator vector layout mismatch");
        if (in.dtype != m.dtype || out.dtype != m.dtype)
            fail(OWTK_ERR_INVALID_ARGUMENT, "vector dtype differs from operator dtype");
        host_apply_call(*m.ctx, m.host_apply, m.host_user, m.host_in, m.host_out, in, out);
        return;
    }
    if (m.dtype == OWTK_F64) {
        matrix_layout_check<double>(m, in, out);
        kern::spmv<double>(*m.ctx, m, static_cast<const double*>(in.data), static_cast<double*>(out.data));
    } else {
        matrix_layout_check<float>(m, in, out);
        kern::spmv<float>(*m.ctx, m, static_cast<const float*>(in.data), static_cast<float*>(out.data));
    }
}

void mixed_apply(Preconditioner& p, Vector& in, Vector& out);

void matrix_layout_check_f64(Matrix& m, Vector& in, Vector& out) { matrix_layout_check<double>(m, in, out); }

bool apply_preconditioner_product(Preconditioner* p, Vector& in, Vector& out, double* product)
{
    if (p == nullptr || p->kind != OWTK_PC_LEARNED) {
        apply_preconditioner(p, in, out);
        return false;
    }
    if (!in.same_layout(out) || in.owned != p->owned || in.ghost != p->ghost || in.bs != p->bs)
        fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner layout mismatch");
    if (in.dtype != OWTK_F64 || out.dtype != OWTK_F64)
        fail(OWTK_ERR_INVALID_ARGUMENT, "the learned preconditioner applies to FP64 vectors");
    return learned_apply(*p, in, out, product);
}

void apply_preconditioner(Preconditioner* p, Vector& in, Vector& out)
{
    if (!in.same_layout(out)) fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner layout mismatch");
    Context& c = *in.ctx;
    const std::size_t n = in.owned_size();
    if (p != nullptr && p->kind == OWTK_PC_LEARNED) {
        if (in.owned != p->owned || in.ghost != p->ghost || in.bs != p->bs)
            fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner layout mismatch");
        if (in.dtype != OWTK_F64 || out.dtype != OWTK_F64)
            fail(OWTK_ERR_INVALID_ARGUMENT, "the learned preconditioner applies to FP64 vectors");
        learned_apply(*p, in, out);
        return;
    }
    if (p != nullptr && (p->kind == OWTK_PC_MIXED || p->storage != OWTK_F64 || p->block)) {
        if (in.owned != p->owned || in.ghost != p->ghost || in.bs != p->bs)
            fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner layout mismatch");
        const owtk_dtype want = (p->kind == OWTK_PC_MIXED || p->storage == OWTK_F64) ? OWTK_F64 : OWTK_F32;
        if (in.dtype != want || out.dtype != want)
            fail(OWTK_ERR_INVALID_ARGUMENT, want == OWTK_F32 ? "stored-precision factors apply to FP32 vectors"
                                                             : "this preconditioner applies to FP64 vectors");
        if (p->kind == OWTK_PC_MIXED) mixed_apply(*p, in, out);
        else if (p->storage == OWTK_F32)
            kern::ilu_apply_lp<float>(c, *p, static_cast<const float*>(in.data), static_cast<float*>(out.data));
        else if (p->storage == OWTK_BF16)
            kern::ilu_apply_lp<__nv_bfloat16>(c, *p, static_cast<const float*>(in.data), static_cast<float*>(out.data));
        else
            kern::block_ilu_apply(c, *p, static_cast<const double*>(in.data), static_cast<double*>(out.data));
        return;
    }
    if (p != nullptr && p->kind == OWTK_PC_CALLBACK) {
        if (in.owned != p->owned || in.ghost != p->ghost || in.bs != p->bs)
            fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner layout mismatch");
        if (in.dtype != p->dtype || out.dtype != p->dtype)
            fail(OWTK_ERR_INVALID_ARGUMENT, "vector dtype differs from preconditioner dtype");
        host_apply_call(c, p->host_apply, p->host_user, p->host_in, p->host_out, in, out);
        return;
    }
    if (p == nullptr || p->kind == OWTK_PC_IDENTITY) {
        if (in.dtype == OWTK_F64) kern::copy<double>(c, n, static_cast<const double*>(in.data), static_cast<double*>(out.data));
        else kern::copy<float>(c, n, static_cast<const float*>(in.data), static_cast<float*>(out.data));
        return;
    }
    if (in.owned != p->owned || in.ghost != p->ghost || in.bs != p->bs)
        fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner layout mismatch");
    if (in.dtype != p->dtype || out.dtype != p->dtype)
        fail(OWTK_ERR_INVALID_ARGUMENT, "vector dtype differs from preconditioner dtype");
    auto run = [&](auto tag) {
        using T = decltype(tag);
        const T* x = static_cast<const T*>(in.data);
        T* y = static_cast<T*>(out.data);
        switch (p->kind) {
        case OWTK_PC_JACOBI: kern::jacobi<T>(c, n, p->inv_diag.as<T>(), x, y); break;
        case OWTK_PC_SSOR:
        case OWTK_PC_SPLIT_SSOR: kern::ssor_apply<T>(c, *p, x, y); break;
        case OWTK_PC_ILU: kern::ilu_apply<T>(c, *p, x, y); break;
        default: break;
        }
    };
    if (in.dtype == OWTK_F64) run(double{});
    else run(float{});
}

}  // namespace owtk

using namespace owtk;

extern "C" {

const char* owtk_last_error(void) { return g_last_error.c_str(); }
int owtk_abi_version(void) { return 1; }

owtk_status owtk_context_create(int device, owtk_context** out)
{
    return guarded([&] {
        require(out != nullptr, "null output handle");
        int count = 0;
        if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
            fail(OWTK_ERR_NO_DEVICE, "no CUDA device is available");
        require(device >= 0 && device < count, "device index out of range");
        OWTK_CUDA(cudaSetDevice(device));
        auto c = std::make_unique<owtk_context>();
        c->device = device;
        OWTK_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
        OWTK_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        OWTK_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&c->host_scalars), kScalarSlots * sizeof(double),
                                cudaHostAllocMapped));
        OWTK_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&c->dev_scalars), c->host_scalars, 0));
        c->dev_scalar_copy.allocate(kScalarSlots * sizeof(double));
        c->partials.allocate(static_cast<std::size_t>(kReduceBlocks) * (kMaxBatch + 1) * 2 * sizeof(double));
        c->tickets.allocate(64 * sizeof(unsigned));
        c->status.allocate(64 * sizeof(unsigned));
        OWTK_CUDA(cudaMemsetAsync(c->tickets.ptr, 0, 64 * sizeof(unsigned), c->stream));
        OWTK_CUDA(cudaMemsetAsync(c->status.ptr, 0, 64 * sizeof(unsigned), c->stream));
        c->sync();
        *out = c.release();
    });
}

owtk_status owtk_context_destroy(owtk_context* ctx)
{
    return guarded([&] { delete ctx; });
}

owtk_status owtk_context_synchronize(owtk_context* ctx)
{
    return guarded([&] {
        require(ctx != nullptr, "null context");
        ctx->check_device_status();
    });
}

void* owtk_context_stream(owtk_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }
uint64_t owtk_context_kernel_launches(owtk_context* ctx) { return ctx ? ctx->launches : 0; }

// ------------------------------------------------------------ vectors
owtk_status owtk_vector_create(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost,
                               size_t bs, owtk_vector** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        if (owned == 0 || bs == 0) fail(OWTK_ERR_INVALID_ARGUMENT, "invalid BlockVector layout or storage size");
        auto v = std::make_unique<owtk_vector>();
        v->ctx = ctx;
        v->dtype = dtype;
        v->owned = owned;
        v->ghost = ghost;
        v->bs = bs;
        v->storage.allocate(v->local_size() * v->elem());
        OWTK_CUDA(cudaMemsetAsync(v->storage.ptr, 0, v->local_size() * v->elem(), ctx->stream));
        v->data = v->storage.ptr;
        *out = v.release();
    });
}

owtk_status owtk_vector_view(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost,
                             size_t bs, void* device_values, size_t value_count, owtk_vector** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        if (owned == 0 || bs == 0 || value_count != (owned + ghost) * bs || device_values == nullptr)
            fail(OWTK_ERR_INVALID_ARGUMENT, "invalid BlockVector layout or storage size");
        auto v = std::make_unique<owtk_vector>();
        v->ctx = ctx;
        v->dtype = dtype;
        v->owned = owned;
        v->ghost = ghost;
        v->bs = bs;
        v->data = device_values;
        v->is_view = true;
        *out = v.release();
    });
}

owtk_status owtk_vector_destroy(owtk_vector* v)
{
    return guarded([&] { delete v; });
}

void* owtk_vector_data(owtk_vector* v) { return v ? v->data : nullptr; }

owtk_status owtk_vector_upload(owtk_vector* v, const void* host, size_t count)
{
    return guarded([&] {
        require(v != nullptr && (host != nullptr || count == 0), "null handle");
        if (count > v->local_size()) fail(OWTK_ERR_OUT_OF_RANGE, "upload larger than the vector");
        OWTK_CUDA(cudaMemcpyAsync(v->data, host, count * v->elem(), cudaMemcpyHostToDevice, v->ctx->stream));
        v->ctx->sync();
    });
}

owtk_status owtk_vector_download(owtk_vector* v, void* host, size_t count)
{
    return guarded([&] {
        require(v != nullptr && (host != nullptr || count == 0), "null handle");
        if (count > v->local_size()) fail(OWTK_ERR_OUT_OF_RANGE, "download larger than the vector");
        OWTK_CUDA(cudaMemcpyAsync(host, v->data, count * v->elem(), cudaMemcpyDeviceToHost, v->ctx->stream));
        v->ctx->sync();
    });
}

owtk_status owtk_vector_fill(owtk_vector* v, double value, int owned_only)
{
    return guarded([&] {
        require(v != nullptr, "null handle");
        const std::size_t n = owned_only ? v->owned_size() : v->local_size();
        if (v->dtype == OWTK_F64) kern::fill<double>(*v->ctx, n, value, static_cast<double*>(v->data));
        else kern::fill<float>(*v->ctx, n, static_cast<float>(value), static_cast<float*>(v->data));
    });
}

// ------------------------------------------------------------ BLAS-1
namespace {
void same_layout_or_throw(const Vector* a, const Vector* b)
{
    require(a != nullptr && b != nullptr, "null handle");
    if (!a->same_layout(*b) || a->dtype != b->dtype)
        fail(OWTK_ERR_INVALID_ARGUMENT, "BlockVector layout mismatch");
}
}  // namespace

owtk_status owtk_copy_owned(owtk_vector* src, owtk_vector* dst)
{
    return guarded([&] {
        same_layout_or_throw(src, dst);
        if (src->dtype == OWTK_F64) kern::copy<double>(*src->ctx, src->owned_size(), static_cast<const double*>(src->data), static_cast<double*>(dst->data));
        else kern::copy<float>(*src->ctx, src->owned_size(), static_cast<const float*>(src->data), static_cast<float*>(dst->data));
    });
}

owtk_status owtk_axpy(double alpha, owtk_vector* x, owtk_vector* y)
{
    return guarded([&] {
        same_layout_or_throw(x, y);
        if (x->dtype == OWTK_F64) kern::axpy<double>(*x->ctx, x->owned_size(), alpha, static_cast<const double*>(x->data), static_cast<double*>(y->data));
        else kern::axpy<float>(*x->ctx, x->owned_size(), static_cast<float>(alpha), static_cast<const float*>(x->data), static_cast<float*>(y->data));
    });
}

owtk_status owtk_scale(double alpha, owtk_vector* x)
{
    return guarded([&] {
        require(x != nullptr, "null handle");
        if (x->dtype == OWTK_F64) kern::scale<double>(*x->ctx, x->owned_size(), alpha, static_cast<double*>(x->data));
        else kern::scale<float>(*x->ctx, x->owned_size(), static_cast<float>(alpha), static_cast<float*>(x->data));
    });
}

owtk_status owtk_assign_linear_combination(owtk_vector* out, double alpha, owtk_vector* x, double beta,
                                           owtk_vector* y)
{
    return guarded([&] {
        same_layout_or_throw(out, x);
        same_layout_or_throw(out, y);
        if (x->dtype == OWTK_F64)
            kern::lincomb<double>(*x->ctx, x->owned_size(), alpha, static_cast<const double*>(x->data), beta,
                                  static_cast<const double*>(y->data), static_cast<double*>(out->data));
        else
            kern::lincomb<float>(*x->ctx, x->owned_size(), static_cast<float>(alpha), static_cast<const float*>(x->data),
                                 static_cast<float>(beta), static_cast<const float*>(y->data), static_cast<float*>(out->data));
    });
}

owtk_status owtk_dot(owtk_vector* a, owtk_vector* b, double* result)
{
    return guarded([&] {
        same_layout_or_throw(a, b);
        require(result != nullptr, "null output");
        Context& c = *a->ctx;
        const void* pa[1] = {a->data};
        const void* pb[1] = {b->data};
        if (a->dtype == OWTK_F64)
            kern::multidot<double>(c, a->owned_size(), 1, reinterpret_cast<const double* const*>(pa),
                                   reinterpret_cast<const double* const*>(pb), c.dev_scalar_copy.as<double>(), c.dev_scalars);
        else
            kern::multidot<float>(c, a->owned_size(), 1, reinterpret_cast<const float* const*>(pa),
                                  reinterpret_cast<const float* const*>(pb), c.dev_scalar_copy.as<double>(), c.dev_scalars);
        c.sync();
        *result = a->dtype == OWTK_F64 ? c.host_scalars[0] : static_cast<double>(static_cast<float>(c.host_scalars[0]));
    });
}

owtk_status owtk_norm(owtk_vector* a, double* result)
{
    return guarded([&] {
        require(a != nullptr && result != nullptr, "null handle");
        Context& c = *a->ctx;
        if (a->dtype == OWTK_F64) kern::norm<double>(c, a->owned_size(), static_cast<const double*>(a->data), c.dev_scalar_copy.as<double>(), c.dev_scalars);
        else kern::norm<float>(c, a->owned_size(), static_cast<const float*>(a->data), c.dev_scalar_copy.as<double>(), c.dev_scalars);
        c.sync();
        *result = a->dtype == OWTK_F64 ? c.host_scalars[0] : static_cast<double>(static_cast<float>(c.host_scalars[0]));
    });
}

owtk_status owtk_dot_batch(owtk_vector* w, owtk_vector* const* basis, size_t k, double* results)
{
    return guarded([&] {
        require(w != nullptr && results != nullptr && (basis != nullptr || k == 0), "null handle");
        if (k + 1 > static_cast<std::size_t>(kMaxBatch)) fail(OWTK_ERR_INVALID_ARGUMENT, "dot batch too large");
        const void* pa[kMaxBatch];
        const void* pb[kMaxBatch];
        for (std::size_t j = 0; j < k; ++j) {
            same_layout_or_throw(w, basis[j]);
            pa[j] = w->data;
            pb[j] = basis[j]->data;
        }
        pa[k] = w->data;
        pb[k] = w->data;
        Context& c = *w->ctx;
        if (w->dtype == OWTK_F64)
            kern::multidot<double>(c, w->owned_size(), static_cast<int>(k + 1), reinterpret_cast<const double* const*>(pa),
                                   reinterpret_cast<const double* const*>(pb), c.dev_scalar_copy.as<double>(), c.dev_scalars);
        else
            kern::multidot<float>(c, w->owned_size(), static_cast<int>(k + 1), reinterpret_cast<const float* const*>(pa),
                                  reinterpret_cast<const float* const*>(pb), c.dev_scalar_copy.as<double>(), c.dev_scalars);
        c.sync();
        for (std::size_t j = 0; j <= k; ++j) results[j] = c.host_scalars[j];
    });
}

// ------------------------------------------------------------ matrices
owtk_status owtk_bsr_create(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost, size_t bs,
                            const uint64_t* rowptr, const uint64_t* cols, const void* values,
                            owtk_matrix** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        if (owned == 0 || bs == 0 || rowptr == nullptr || values == nullptr)
            fail(OWTK_ERR_INVALID_ARGUMENT, "invalid BlockCsrMatrix storage");
        auto m = std::make_unique<owtk_matrix>();
        m->ctx = ctx;
        m->kind = 0;
        m->dtype = dtype;
        ingest_structure(*m, owned, ghost, bs, rowptr, cols, "invalid BlockCsrMatrix storage");
        const std::size_t bytes = m->entries * bs * dsize(dtype);
        m->values.allocate(bytes + 16);
        OWTK_CUDA(cudaMemcpyAsync(m->values.ptr, values, bytes, cudaMemcpyHostToDevice, ctx->stream));
        kern::slices_fill(*ctx, *m);
        ctx->sync();
        *out = m.release();
    });
}

owtk_status owtk_bsr_update_values(owtk_matrix* m, const void* values)
{
    return guarded([&] {
        require(m != nullptr && values != nullptr, "null handle");
        require(m->kind != 1, "split views borrow their coefficients; write the device arrays directly");
        require(m->kind != 3, "a callback operator has no stored values");
        const std::size_t per = m->kind == 2 ? m->bs * m->bs : m->bs;
        OWTK_CUDA(cudaMemcpyAsync(m->values.ptr, values, m->entries * per * dsize(m->dtype),
                                  cudaMemcpyHostToDevice, m->ctx->stream));
        kern::slices_fill(*m->ctx, *m);
        m->ctx->sync();
    });
}

owtk_status owtk_split_view_create(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost, size_t bs,
                                   const uint64_t* rowptr, const uint64_t* cols, const void* device_diagonal,
                                   const void* device_off_diagonal, owtk_matrix** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        if (owned == 0 || bs == 0 || rowptr == nullptr || device_diagonal == nullptr
            || (device_off_diagonal == nullptr && rowptr[owned] != 0))
            fail(OWTK_ERR_INVALID_ARGUMENT, "invalid split CSR storage");
        const auto misaligned = [&](const void* p) {
            return reinterpret_cast<std::uintptr_t>(p) % dsize(dtype) != 0;
        };
        if (misaligned(device_diagonal) || misaligned(device_off_diagonal))
            fail(OWTK_ERR_INVALID_ARGUMENT, "split coefficients are not aligned to their element size");
        auto m = std::make_unique<owtk_matrix>();
        m->ctx = ctx;
        m->kind = 1;
        m->dtype = dtype;
        ingest_structure(*m, owned, ghost, bs, rowptr, cols, "invalid split CSR storage");
        m->diag = device_diagonal;
        m->off = device_off_diagonal;
        ctx->sync();
        *out = m.release();
    });
}

owtk_status owtk_dense_bsr_create(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost, size_t bs,
                                  const uint64_t* rowptr, const uint64_t* cols, const void* values,
                                  owtk_matrix** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        if (owned == 0 || bs == 0 || rowptr == nullptr || values == nullptr)
            fail(OWTK_ERR_INVALID_ARGUMENT, "invalid dense-block CSR storage");
        auto m = std::make_unique<owtk_matrix>();
        m->ctx = ctx;
        m->kind = 2;
        m->dtype = dtype;
        ingest_structure(*m, owned, ghost, bs, rowptr, cols, "invalid dense-block CSR storage");
        const std::size_t bytes = m->entries * bs * bs * dsize(dtype);
        m->values.allocate(bytes + 16);
        OWTK_CUDA(cudaMemcpyAsync(m->values.ptr, values, bytes, cudaMemcpyHostToDevice, ctx->stream));
        kern::slices_fill(*ctx, *m);
        ctx->sync();
        *out = m.release();
    });
}

owtk_status owtk_matrix_destroy(owtk_matrix* m)
{
    return guarded([&] { delete m; });
}

owtk_status owtk_matrix_info(owtk_matrix* m, int* kind, size_t* owned, size_t* ghost, size_t* bs,
                             size_t* entries)
{
    return guarded([&] {
        require(m != nullptr, "null handle");
        if (kind) *kind = m->kind;
        if (owned) *owned = m->owned;
        if (ghost) *ghost = m->ghost;
        if (bs) *bs = m->bs;
        if (entries) *entries = m->kind == 1 ? m->owned + m->entries : m->entries;
    });
}

owtk_status owtk_spmv(owtk_matrix* m, owtk_vector* in, owtk_vector* out)
{
    return guarded([&] {
        require(m != nullptr && in != nullptr && out != nullptr, "null handle");
        apply_operator(*m, *in, *out);
    });
}

owtk_status owtk_spmv_rows(owtk_matrix* m, owtk_vector* in, owtk_vector* out, const uint64_t* host_rows,
                           size_t count)
{
    return guarded([&] {
        require(m != nullptr && in != nullptr && out != nullptr && (host_rows != nullptr || count == 0),
                "null handle");
        if (m->kind == 3) fail(OWTK_ERR_INVALID_ARGUMENT, "a callback operator has no apply_rows()");
        if (m->dtype == OWTK_F64) matrix_layout_check<double>(*m, *in, *out);
        else matrix_layout_check<float>(*m, *in, *out);
        if (count == 0) return;
        require(count <= static_cast<size_t>(INT32_MAX), "too many rows");
        std::vector<std::int32_t> rows(count);
        for (size_t i = 0; i < count; ++i) {
            if (host_rows[i] >= m->owned) fail(OWTK_ERR_OUT_OF_RANGE, "apply_rows: row out of range");
            rows[i] = static_cast<std::int32_t>(host_rows[i]);
        }
        Context& c = *m->ctx;
        const std::size_t bytes = count * sizeof(std::int32_t);
        if (m->row_list.bytes < bytes) m->row_list.allocate(bytes);
        // The previous call's kernel may still read the list: copy behind it
        // on the same stream (pageable source: the copy returns once staged).
        OWTK_CUDA(cudaMemcpyAsync(m->row_list.ptr, rows.data(), bytes, cudaMemcpyHostToDevice, c.stream));
        const int n = static_cast<int>(count);
        if (m->dtype == OWTK_F64)
            kern::spmv_rows<double>(c, *m, m->row_list.as<int>(), n, static_cast<const double*>(in->data),
                                    static_cast<double*>(out->data));
        else
            kern::spmv_rows<float>(c, *m, m->row_list.as<int>(), n, static_cast<const float*>(in->data),
                                   static_cast<float*>(out->data));
    });
}

owtk_status owtk_matrix_diagonal(owtk_matrix* m, void* host_out)
{
    return guarded([&] {
        require(m != nullptr && host_out != nullptr, "null handle");
        const std::size_t n = m->owned * m->bs;
        Context& c = *m->ctx;
        if (m->kind == 2) fail(OWTK_ERR_INVALID_ARGUMENT, "dense-block CSR has no diagonal()");
        if (m->kind == 3) fail(OWTK_ERR_INVALID_ARGUMENT, "a callback operator has no diagonal()");
        if (m->kind == 1) {
            OWTK_CUDA(cudaMemcpyAsync(host_out, m->diag, n * dsize(m->dtype), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            return;
        }
        DeviceBuffer d(n * dsize(m->dtype) + 16);
        if (m->dtype == OWTK_F64) kern::bsr_diagonal<double>(c, *m, d.as<double>());
        else kern::bsr_diagonal<float>(c, *m, d.as<float>());
        try {
            c.check_device_status();
        } catch (const Error&) {
            fail(OWTK_ERR_INVALID_ARGUMENT, "BlockCsrMatrix row has no diagonal");
        }
        OWTK_CUDA(cudaMemcpyAsync(host_out, d.ptr, n * dsize(m->dtype), cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

// ------------------------------------------------------------ preconditioners
}  // extern "C"

namespace owtk {
namespace {

std::unique_ptr<owtk_preconditioner> make_pc(owtk_matrix* m, owtk_pc_kind kind, double parameter,
                                             owtk_dtype storage)
{
    require(m != nullptr, "null handle");
    auto p = std::make_unique<owtk_preconditioner>();
    p->ctx = m->ctx;
    p->kind = kind;
    p->dtype = m->dtype;
    p->matrix = m;
    p->owned = m->owned;
    p->ghost = m->ghost;
    p->bs = m->bs;
    p->parameter = parameter;
    const std::size_t n = m->owned * m->bs;
    const std::size_t es = dsize(m->dtype);
    switch (kind) {
    case OWTK_PC_IDENTITY: break;
    case OWTK_PC_JACOBI:
        if (m->kind == 2 || m->kind == 3) fail(OWTK_ERR_INVALID_ARGUMENT, "Jacobi needs a matrix with diagonal()");
        p->inv_diag.allocate(n * es + 16);
        break;
    case OWTK_PC_SSOR:
    case OWTK_PC_SPLIT_SSOR: {
        if (kind == OWTK_PC_SSOR && m->kind != 0)
            fail(OWTK_ERR_INVALID_ARGUMENT, "SSOR needs a component-diagonal BSR matrix");
        if (kind == OWTK_PC_SPLIT_SSOR && m->kind != 1)
            fail(OWTK_ERR_INVALID_ARGUMENT, "split SSOR needs a split view");
        if (!(parameter > 0 && parameter < 2))
            fail(OWTK_ERR_INVALID_ARGUMENT, kind == OWTK_PC_SSOR ? "SSOR omega must be in (0,2)"
                                                                 : "split SSOR omega must be in (0,2)");
        p->work.allocate(m->local_size() * es + 16);
        if (kind == OWTK_PC_SSOR) p->diag_cache.allocate(n * es + 16);
        std::vector<std::int32_t> lower, upper;
        // The matrix pattern itself is the dependency pattern (ghosts excluded).
        std::vector<std::int32_t> cols = m->h_cols;
        for (auto& c : cols)
            if (static_cast<std::size_t>(c) >= m->owned) c = static_cast<std::int32_t>(m->owned);
        levels_of(m->owned, m->h_rowptr.data(), cols.data(), lower, upper);
        build_sweep(*p->ctx, p->lower, m->owned, m->bs, lower, false);
        build_sweep(*p->ctx, p->upper, m->owned, m->bs, upper, true);
        break;
    }
    case OWTK_PC_ILU: {
        if (m->kind != 0) fail(OWTK_ERR_INVALID_ARGUMENT, "ILU needs a component-diagonal BSR matrix");
        if (!(parameter >= 0)) fail(OWTK_ERR_INVALID_ARGUMENT, "ILU fill level must be >= 0");
        ilu_symbolic(*p, *m, static_cast<std::size_t>(parameter));
        if (storage == OWTK_F64 && m->bs <= 32 && !p->chain.ready) {
            const char* env = std::getenv("OWTK_PACKED_SWEEP");   // 0: applies read the factor in place
            if (!env || std::atoi(env) != 0) {
                pack_sweep(*p->ctx, p->lower, m->bs, es, p->f_rowptr, p->f_cols, p->f_diagpos, false);
                pack_sweep(*p->ctx, p->upper, m->bs, es, p->f_rowptr, p->f_cols, p->f_diagpos, true);
            }
        }
        break;
    }
    case OWTK_PC_BLOCK_ILU: {
        if (m->kind != 2) fail(OWTK_ERR_INVALID_ARGUMENT, "block ILU needs a dense-block BSR matrix");
        if (m->dtype != OWTK_F64) fail(OWTK_ERR_INVALID_ARGUMENT, "block ILU factorises an FP64 matrix");
        if (m->bs > 4) fail(OWTK_ERR_INVALID_ARGUMENT, "block ILU supports block sizes up to 4");
        p->block = true;
        ilu_symbolic(*p, *m, 0);
        break;
    }
    default: fail(OWTK_ERR_INVALID_ARGUMENT, "unknown preconditioner kind");
    }
    if (storage != OWTK_F64) {
        if (kind != OWTK_PC_ILU && kind != OWTK_PC_BLOCK_ILU)
            fail(OWTK_ERR_INVALID_ARGUMENT, "stored-precision factors exist for ILU and block ILU only");
        if (m->dtype != OWTK_F64) fail(OWTK_ERR_INVALID_ARGUMENT, "stored-precision factors come from an FP64 matrix");
        if (storage != OWTK_F32 && storage != OWTK_BF16) fail(OWTK_ERR_INVALID_ARGUMENT, "storage must be F32 or BF16");
        p->storage = storage;
        const std::size_t per = p->block ? m->bs * m->bs : m->bs;
        p->lp_vals.allocate(p->f_cols.size() * per * dsize(storage) + 16);
        p->lp_inv.allocate(m->owned * per * dsize(storage) + 16);
        p->work32.allocate(n * sizeof(float) + 16);
    }
    if (kind == OWTK_PC_SSOR || kind == OWTK_PC_SPLIT_SSOR || kind == OWTK_PC_ILU || kind == OWTK_PC_BLOCK_ILU) {
        p->flags.allocate(m->owned * sizeof(unsigned) + 16);
        OWTK_CUDA(cudaMemsetAsync(p->flags.ptr, 0, m->owned * sizeof(unsigned), p->ctx->stream));
        p->ticket.allocate(sizeof(unsigned long long));
        OWTK_CUDA(cudaMemsetAsync(p->ticket.ptr, 0, sizeof(unsigned long long), p->ctx->stream));
    }
    if (kind != OWTK_PC_IDENTITY) numeric_update(*p, *m);
    p->ctx->sync();
    return p;
}

// FP32 copy of an FP64 owning matrix (structure shared by value, values
// converted on the device by the mixed preconditioner's numeric update).
std::unique_ptr<Matrix> f32_copy(const Matrix& m)
{
    if (m.kind == 1 || m.kind == 3)
        fail(OWTK_ERR_INVALID_ARGUMENT, "mixed precision needs an owning matrix, not a split view or callback");
    auto c = std::make_unique<owtk_matrix>();
    c->ctx = m.ctx;
    c->kind = m.kind;
    c->dtype = OWTK_F32;
    c->owned = m.owned;
    c->ghost = m.ghost;
    c->bs = m.bs;
    c->entries = m.entries;
    c->h_rowptr = m.h_rowptr;
    c->h_cols = m.h_cols;
    c->rowptr = upload(m.ctx->stream, c->h_rowptr);
    c->cols = upload(m.ctx->stream, c->h_cols);
    build_tile_plan(*c);
    const std::size_t per = m.kind == 2 ? m.bs * m.bs : m.bs;
    c->values.allocate(m.entries * per * sizeof(float) + 16);
    return c;
}

}  // namespace

// FP64 in/out through an FP32 inner solve (owtk_pc_create_mixed).
void mixed_apply(Preconditioner& p, Vector& in, Vector& out)
{
    Context& c = *p.ctx;
    const std::size_t n = p.owned * p.bs;
    owtk_vector vin, vout;
    for (owtk_vector* v : {&vin, &vout}) {
        v->ctx = p.ctx;
        v->dtype = OWTK_F32;
        v->owned = p.owned;
        v->ghost = p.ghost;
        v->bs = p.bs;
        v->is_view = true;
    }
    vin.data = p.v32.ptr;
    vout.data = p.z32.ptr;
    kern::convert<float, double>(c, n, static_cast<const double*>(in.data), p.v32.as<float>());
    if (p.inner_iterations == 0) {
        apply_preconditioner(p.inner.get(), vin, vout);
    } else {
        kern::fill<float>(c, vout.local_size(), 0.0f, p.z32.as<float>());
        owtk_solver_options o;
        owtk_default_options(&o);
        o.restart = p.inner_iterations;
        o.maximum_iterations = p.inner_iterations;
        o.relative_tolerance = 0;
        o.absolute_tolerance = 0;
        owtk_solver_result r;
        solve(OWTK_SOLVER_FGMRES, *p.m32, p.inner.get(), vin, vout, o, *p.inner_ws, r);
    }
    kern::convert<double, float>(c, n, p.z32.as<float>(), static_cast<double*>(out.data));
}

}  // namespace owtk

extern "C" {

owtk_status owtk_pc_create(owtk_matrix* m, owtk_pc_kind kind, double parameter, owtk_preconditioner** out)
{
    return guarded([&] {
        require(m != nullptr && out != nullptr, "null handle");
        if (kind == OWTK_PC_MIXED) fail(OWTK_ERR_INVALID_ARGUMENT, "use owtk_pc_create_mixed");
        *out = make_pc(m, kind, parameter, OWTK_F64).release();
    });
}

owtk_status owtk_pc_create_stored(owtk_matrix* m, owtk_pc_kind kind, double parameter, owtk_dtype storage,
                                  owtk_preconditioner** out)
{
    return guarded([&] {
        require(m != nullptr && out != nullptr, "null handle");
        *out = make_pc(m, kind, parameter, storage).release();
    });
}

owtk_status owtk_pc_create_mixed(owtk_matrix* m, owtk_pc_kind inner_kind, double parameter, owtk_dtype storage,
                                 uint32_t inner_iterations, owtk_preconditioner** out)
{
    return guarded([&] {
        require(m != nullptr && out != nullptr, "null handle");
        if (m->dtype != OWTK_F64) fail(OWTK_ERR_INVALID_ARGUMENT, "the mixed preconditioner serves FP64 solves");
        if (storage == OWTK_F64) fail(OWTK_ERR_INVALID_ARGUMENT, "mixed precision stores factors in F32 or BF16");
        auto p = std::make_unique<owtk_preconditioner>();
        p->ctx = m->ctx;
        p->kind = OWTK_PC_MIXED;
        p->dtype = OWTK_F64;
        p->matrix = m;
        p->owned = m->owned;
        p->ghost = m->ghost;
        p->bs = m->bs;
        p->parameter = parameter;
        p->storage = storage;
        p->inner_iterations = inner_iterations;
        p->m32 = f32_copy(*m);
        p->inner = make_pc(m, inner_kind, parameter, storage);
        p->inner_ws = std::make_unique<Workspace>();
        p->inner_ws->ctx = m->ctx;
        p->v32.allocate(m->local_size() * sizeof(float) + 16);
        p->z32.allocate(m->local_size() * sizeof(float) + 16);
        OWTK_CUDA(cudaMemsetAsync(p->v32.ptr, 0, m->local_size() * sizeof(float), m->ctx->stream));
        const std::size_t per = m->kind == 2 ? m->bs * m->bs : m->bs;
        kern::convert<float, double>(*m->ctx, m->entries * per, m->values.as<double>(), p->m32->values.as<float>());
        kern::slices_fill(*m->ctx, *p->m32);
        p->numeric_updates = 1;
        m->ctx->sync();
        *out = p.release();
    });
}

owtk_status owtk_pc_destroy(owtk_preconditioner* pc)
{
    return guarded([&] { delete pc; });
}

owtk_status owtk_pc_apply(owtk_preconditioner* pc, owtk_vector* in, owtk_vector* out)
{
    return guarded([&] {
        require(pc != nullptr && in != nullptr && out != nullptr, "null handle");
        apply_preconditioner(pc, *in, *out);
    });
}

owtk_status owtk_pc_update_values(owtk_preconditioner* pc, owtk_matrix* m)
{
    return guarded([&] {
        require(pc != nullptr && m != nullptr, "null handle");
        if (m->owned != pc->owned || m->ghost != pc->ghost || m->bs != pc->bs || m->dtype != pc->dtype)
            fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner matrix layout mismatch");
        if (pc->kind == OWTK_PC_CALLBACK)
            fail(OWTK_ERR_INVALID_ARGUMENT, "a callback preconditioner has no numeric values to update");
        if (pc->kind == OWTK_PC_ILU || pc->kind == OWTK_PC_BLOCK_ILU) ilu_pattern_check(*pc, *m);
        if (pc->kind == OWTK_PC_MIXED) {
            if (m->kind != pc->m32->kind) fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner matrix kind mismatch");
            ilu_pattern_check(*pc->inner, *m);
            pc->inner->matrix = m;
        }
        if ((pc->kind == OWTK_PC_SSOR || pc->kind == OWTK_PC_SPLIT_SSOR) && m != pc->matrix)
            fail(OWTK_ERR_INVALID_ARGUMENT, "SSOR refreshes from the matrix it was built on");
        pc->matrix = m;
        if (pc->kind != OWTK_PC_IDENTITY) numeric_update(*pc, *m);
    });
}

uint64_t owtk_pc_numeric_updates(owtk_preconditioner* pc) { return pc ? pc->numeric_updates : 0; }

owtk_status owtk_ilu_factors(owtk_preconditioner* pc, uint64_t* entries, uint64_t* rowptr, uint64_t* cols,
                             void* values, void* inverse_diagonal)
{
    return guarded([&] {
        require(pc != nullptr && entries != nullptr, "null handle");
        if (pc->kind != OWTK_PC_ILU && pc->kind != OWTK_PC_BLOCK_ILU)
            fail(OWTK_ERR_INVALID_ARGUMENT, "not an ILU preconditioner");
        *entries = pc->f_cols.size();
        const std::size_t per = pc->block ? pc->bs * pc->bs : pc->bs;
        if (rowptr) for (std::size_t i = 0; i < pc->f_rowptr.size(); ++i) rowptr[i] = static_cast<std::uint64_t>(pc->f_rowptr[i]);
        if (cols) for (std::size_t i = 0; i < pc->f_cols.size(); ++i) cols[i] = static_cast<std::uint64_t>(pc->f_cols[i]);
        const std::size_t es = dsize(pc->dtype);
        if (values)
            OWTK_CUDA(cudaMemcpyAsync(values, pc->d_fvalues.ptr, pc->f_cols.size() * per * es, cudaMemcpyDeviceToHost, pc->ctx->stream));
        if (inverse_diagonal)
            OWTK_CUDA(cudaMemcpyAsync(inverse_diagonal, pc->inv_diag.ptr, pc->owned * per * es, cudaMemcpyDeviceToHost, pc->ctx->stream));
        pc->ctx->sync();
    });
}

owtk_status owtk_pc_levels(owtk_preconditioner* pc, int32_t* lower, int32_t* upper, uint64_t* lower_depth,
                           uint64_t* upper_depth)
{
    return guarded([&] {
        require(pc != nullptr, "null handle");
        if (pc->kind != OWTK_PC_ILU && pc->kind != OWTK_PC_SSOR && pc->kind != OWTK_PC_SPLIT_SSOR
            && pc->kind != OWTK_PC_BLOCK_ILU)
            fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner has no sweep schedule");
        if (lower) std::copy(pc->lower.h_level.begin(), pc->lower.h_level.end(), lower);
        if (upper) std::copy(pc->upper.h_level.begin(), pc->upper.h_level.end(), upper);
        if (lower_depth) *lower_depth = static_cast<std::uint64_t>(pc->lower.depth);
        if (upper_depth) *upper_depth = static_cast<std::uint64_t>(pc->upper.depth);
    });
}

// ------------------------------------------------------------ orderings
namespace {
void narrow_pattern(std::size_t owned, std::size_t ghost, const uint64_t* rowptr, const uint64_t* cols,
                    std::vector<std::int32_t>& rp, std::vector<std::int32_t>& ci)
{
    require(rowptr != nullptr && (cols != nullptr || rowptr[owned] == 0), "null pattern");
    require(owned + ghost < static_cast<std::size_t>(std::numeric_limits<std::int32_t>::max())
                && rowptr[owned] < static_cast<std::uint64_t>(std::numeric_limits<std::int32_t>::max()),
            "pattern too large for 32-bit indices");
    rp.resize(owned + 1);
    for (std::size_t r = 0; r <= owned; ++r) rp[r] = static_cast<std::int32_t>(rowptr[r]);
    ci.resize(rowptr[owned]);
    for (std::size_t e = 0; e < ci.size(); ++e) {
        if (cols[e] >= owned + ghost) fail(OWTK_ERR_INVALID_ARGUMENT, "column outside local layout");
        ci[e] = static_cast<std::int32_t>(cols[e]);
    }
}
}  // namespace

owtk_status owtk_rcm_order(size_t owned, size_t ghost, const uint64_t* rowptr, const uint64_t* cols,
                           uint64_t* new_to_old)
{
    return guarded([&] {
        require(new_to_old != nullptr, "null output");
        std::vector<std::int32_t> rp, ci;
        narrow_pattern(owned, ghost, rowptr, cols, rp, ci);
        rcm_order(owned, rp.data(), ci.data(), new_to_old);
    });
}

owtk_status owtk_hilbert_order(size_t n, const double* xy, uint64_t* new_to_old)
{
    return guarded([&] {
        require((xy != nullptr && new_to_old != nullptr) || n == 0, "null pointer");
        hilbert_order(n, xy, new_to_old);
    });
}

owtk_status owtk_inverse_permutation(size_t n, const uint64_t* in, uint64_t* out)
{
    return guarded([&] {
        require((in != nullptr && out != nullptr) || n == 0, "null pointer");
        std::vector<char> seen(n, 0);
        for (std::size_t i = 0; i < n; ++i) {
            const std::uint64_t o = in[i];
            if (o >= n || seen[o]) fail(OWTK_ERR_INVALID_ARGUMENT, "invalid node permutation");
            seen[o] = 1;
            out[o] = i;
        }
    });
}

owtk_status owtk_level_sets(size_t owned, const uint64_t* rowptr, const uint64_t* cols, int32_t* lower,
                            int32_t* upper, uint64_t* lower_depth, uint64_t* upper_depth)
{
    return guarded([&] {
        std::vector<std::int32_t> rp, ci;
        narrow_pattern(owned, std::numeric_limits<std::int32_t>::max() / 2 - owned, rowptr, cols, rp, ci);
        for (auto& c : ci)
            if (static_cast<std::size_t>(c) >= owned) c = static_cast<std::int32_t>(owned);
        std::vector<std::int32_t> lo, up;
        levels_of(owned, rp.data(), ci.data(), lo, up);
        std::int32_t dl = 0, du = 0;
        for (std::size_t r = 0; r < owned; ++r) {
            dl = std::max(dl, lo[r] + 1);
            du = std::max(du, up[r] + 1);
        }
        if (lower) std::copy(lo.begin(), lo.end(), lower);
        if (upper) std::copy(up.begin(), up.end(), upper);
        if (lower_depth) *lower_depth = static_cast<std::uint64_t>(dl);
        if (upper_depth) *upper_depth = static_cast<std::uint64_t>(du);
    });
}

// ------------------------------------------------------------ workspace
owtk_status owtk_workspace_create(owtk_context* ctx, owtk_workspace** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        auto w = std::make_unique<owtk_workspace>();
        w->ctx = ctx;
        *out = w.release();
    });
}

owtk_status owtk_workspace_destroy(owtk_workspace* ws)
{
    return guarded([&] { delete ws; });
}

uint64_t owtk_workspace_allocation_epochs(owtk_workspace* ws) { return ws ? ws->epochs : 0; }

// ------------------------------------------------------------ permutations
owtk_status owtk_permutation_create(owtk_context* ctx, size_t n, const uint64_t* new_to_old, owtk_permutation** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr && new_to_old != nullptr && n > 0, "null handle or empty permutation");
        auto p = std::make_unique<owtk_permutation>();
        p->ctx = ctx;
        p->n = n;
        p->new_to_old.resize(n);
        p->old_to_new.assign(n, -1);
        // ordering.hpp:263-277: every index exactly once.
        for (std::size_t i = 0; i < n; ++i) {
            if (new_to_old[i] >= n || p->old_to_new[new_to_old[i]] != -1)
                fail(OWTK_ERR_INVALID_ARGUMENT, "invalid permutation");
            p->new_to_old[i] = static_cast<std::int64_t>(new_to_old[i]);
            p->old_to_new[new_to_old[i]] = static_cast<std::int64_t>(i);
        }
        p->d_new_to_old = upload(ctx->stream, p->new_to_old);
        ctx->sync();
        *out = p.release();
    });
}

owtk_status owtk_permutation_destroy(owtk_permutation* p)
{
    return guarded([&] { delete p; });
}

owtk_status owtk_vector_permute(owtk_permutation* p, owtk_vector* src, owtk_vector* dst, int inverse)
{
    return guarded([&] {
        require(p != nullptr && src != nullptr && dst != nullptr, "null handle");
        same_layout_or_throw(src, dst);
        if (src->owned != p->n) fail(OWTK_ERR_INVALID_ARGUMENT, "permutation size differs from owned nodes");
        if (src->data == dst->data) fail(OWTK_ERR_INVALID_ARGUMENT, "source and destination must differ");
        Context& c = *src->ctx;
        if (src->dtype == OWTK_F64)
            kern::permute_nodes<double>(c, p->n, src->bs, p->d_new_to_old.as<std::int64_t>(),
                                        static_cast<const double*>(src->data), static_cast<double*>(dst->data), inverse != 0);
        else
            kern::permute_nodes<float>(c, p->n, src->bs, p->d_new_to_old.as<std::int64_t>(),
                                       static_cast<const float*>(src->data), static_cast<float*>(dst->data), inverse != 0);
        c.sync();
    });
}

owtk_status owtk_bsr_create_permuted_split(owtk_permutation* p, owtk_dtype dtype, size_t bs,
                                           const uint64_t* off_rowptr, const uint64_t* off_cols,
                                           const void* device_diagonal, const void* device_off_diagonal,
                                           owtk_matrix** out)
{
    return guarded([&] {
        require(p != nullptr && out != nullptr && off_rowptr != nullptr && device_diagonal != nullptr, "null handle");
        if (dtype != OWTK_F64 && dtype != OWTK_F32) fail(OWTK_ERR_INVALID_ARGUMENT, "dtype must be F64 or F32");
        if (bs == 0) fail(OWTK_ERR_INVALID_ARGUMENT, "invalid split CSR storage");
        const std::size_t n = p->n;
        const std::uint64_t edges = off_rowptr[n];
        if (off_rowptr[0] != 0 || (edges > 0 && (off_cols == nullptr || device_off_diagonal == nullptr)))
            fail(OWTK_ERR_INVALID_ARGUMENT, "invalid split CSR storage");
        // New row i is old row new_to_old[i]: its diagonal plus its edges with
        // relabelled columns, sorted by new column.
        std::vector<std::uint64_t> rowptr(n + 1, 0), cols;
        std::vector<std::int64_t> map;
        cols.reserve(n + edges);
        map.reserve(n + edges);
        std::vector<std::pair<std::uint64_t, std::int64_t>> row;
        for (std::size_t i = 0; i < n; ++i) {
            const std::size_t o = static_cast<std::size_t>(p->new_to_old[i]);
            if (off_rowptr[o] > off_rowptr[o + 1]) fail(OWTK_ERR_INVALID_ARGUMENT, "nonmonotone split CSR offsets");
            row.clear();
            row.emplace_back(i, static_cast<std::int64_t>(o));
            for (std::uint64_t k = off_rowptr[o]; k < off_rowptr[o + 1]; ++k) {
                if (off_cols[k] >= n) fail(OWTK_ERR_INVALID_ARGUMENT, "split CSR column outside owned nodes");
                if (off_cols[k] == o) fail(OWTK_ERR_INVALID_ARGUMENT, "split CSR edge on the diagonal");
                row.emplace_back(static_cast<std::uint64_t>(p->old_to_new[off_cols[k]]),
                                 static_cast<std::int64_t>(n + k));
            }
            std::sort(row.begin(), row.end());
            for (const auto& [col, src] : row) {
                cols.push_back(col);
                map.push_back(src);
            }
            rowptr[i + 1] = cols.size();
        }
        auto m = std::make_unique<owtk_matrix>();
        m->ctx = p->ctx;
        m->kind = 0;
        m->dtype = dtype;
        ingest_structure(*m, n, 0, bs, rowptr.data(), cols.data(), "invalid split CSR storage");
        m->values.allocate(m->entries * bs * dsize(dtype) + 16);
        m->split_map = upload(p->ctx->stream, map);
        m->split_edges = edges;
        Context& c = *p->ctx;
        if (dtype == OWTK_F64)
            kern::gather_split<double>(c, m->entries, bs, n, m->split_map.as<std::int64_t>(),
                                       static_cast<const double*>(device_diagonal),
                                       static_cast<const double*>(device_off_diagonal), m->values.as<double>());
        else
            kern::gather_split<float>(c, m->entries, bs, n, m->split_map.as<std::int64_t>(),
                                      static_cast<const float*>(device_diagonal),
                                      static_cast<const float*>(device_off_diagonal), m->values.as<float>());
        kern::slices_fill(c, *m);
        c.sync();
        *out = m.release();
    });
}

owtk_status owtk_bsr_update_permuted_split(owtk_matrix* m, const void* device_diagonal, const void* device_off_diagonal)
{
    return guarded([&] {
        require(m != nullptr && device_diagonal != nullptr, "null handle");
        if (m->split_map.ptr == nullptr)
            fail(OWTK_ERR_INVALID_ARGUMENT, "matrix was not built by owtk_bsr_create_permuted_split");
        if (m->split_edges > 0 && device_off_diagonal == nullptr) fail(OWTK_ERR_INVALID_ARGUMENT, "null off-diagonal");
        Context& c = *m->ctx;
        if (m->dtype == OWTK_F64)
            kern::gather_split<double>(c, m->entries, m->bs, m->owned, m->split_map.as<std::int64_t>(),
                                       static_cast<const double*>(device_diagonal),
                                       static_cast<const double*>(device_off_diagonal), m->values.as<double>());
        else
            kern::gather_split<float>(c, m->entries, m->bs, m->owned, m->split_map.as<std::int64_t>(),
                                      static_cast<const float*>(device_diagonal),
                                      static_cast<const float*>(device_off_diagonal), m->values.as<float>());
        kern::slices_fill(c, *m);
        c.sync();
    });
}

owtk_status owtk_pc_sweep_schedule(owtk_preconditioner* pc, int32_t* cluster_ctas, int32_t* epoch_levels,
                                   int32_t* ring_rows)
{
    return guarded([&] {
        require(pc != nullptr, "null handle");
        const bool on = pc->c_lower.ready && pc->c_upper.ready;
        if (cluster_ctas) *cluster_ctas = on ? pc->c_lower.C : 0;
        if (epoch_levels) *epoch_levels = on ? pc->c_lower.K : 0;
        if (ring_rows) *ring_rows = on ? std::max(pc->c_lower.R, pc->c_upper.R) : 0;
    });
}

owtk_status owtk_pc_lockstep_schedule(owtk_preconditioner* pc, int32_t* cluster_ctas, int32_t* lower_levels,
                                      int32_t* upper_levels)
{
    return guarded([&] {
        require(pc != nullptr, "null handle");
        const bool on = pc->l_lower.ready && pc->l_upper.ready;
        if (cluster_ctas) *cluster_ctas = on ? pc->l_lower.C : 0;
        if (lower_levels) *lower_levels = on ? pc->l_lower.D : 0;
        if (upper_levels) *upper_levels = on ? pc->l_upper.D : 0;
    });
}

owtk_status owtk_pc_chain_schedule(owtk_preconditioner* pc, int32_t* windows)
{
    return guarded([&] {
        require(pc != nullptr, "null handle");
        if (windows) *windows = pc->chain.ready ? pc->chain.count : 0;
    });
}

// ------------------------------------------------------------ bounded waits
owtk_status owtk_debug_unpublished_dependency(owtk_context* ctx, uint32_t spin_limit)
{
    return guarded([&] {
        require(ctx != nullptr && spin_limit > 0 && spin_limit <= (1u << 22), "spin limit out of range");
        kern::debug_unpublished_dependency(*ctx, static_cast<int>(spin_limit));
        ctx->check_device_status();
    });
}

// ------------------------------------------------------------ extras
owtk_status owtk_dot_ex(owtk_vector* a, owtk_vector* b, owtk_reduction_kind reduction, double* result, double* low)
{
    return guarded([&] {
        same_layout_or_throw(a, b);
        require(result != nullptr, "null output");
        if (reduction < OWTK_REDUCTION_SERIAL || reduction > OWTK_REDUCTION_MIXED_PRECISION)
            fail(OWTK_ERR_INVALID_ARGUMENT, "unknown reduction kind");
        Context& c = *a->ctx;
        const void* pa[1] = {a->data};
        const void* pb[1] = {b->data};
        double* lo_slot = c.dev_scalars + 1;   // host view of scalar slot 1
        if (reduction == OWTK_REDUCTION_SERIAL) {
            if (a->dtype == OWTK_F64)
                kern::multidot<double>(c, a->owned_size(), 1, reinterpret_cast<const double* const*>(pa),
                                       reinterpret_cast<const double* const*>(pb), c.dev_scalar_copy.as<double>(),
                                       c.dev_scalars);
            else
                kern::multidot<float>(c, a->owned_size(), 1, reinterpret_cast<const float* const*>(pa),
                                      reinterpret_cast<const float* const*>(pb), c.dev_scalar_copy.as<double>(),
                                      c.dev_scalars);
            c.host_scalars[1] = 0.0;
        } else if (a->dtype == OWTK_F64) {
            kern::multidot_accurate<double>(c, a->owned_size(), 1, reduction, reinterpret_cast<const double* const*>(pa),
                                            reinterpret_cast<const double* const*>(pb), c.dev_scalar_copy.as<double>(),
                                            c.dev_scalars, lo_slot);
        } else {
            kern::multidot_accurate<float>(c, a->owned_size(), 1, reduction, reinterpret_cast<const float* const*>(pa),
                                           reinterpret_cast<const float* const*>(pb), c.dev_scalar_copy.as<double>(),
                                           c.dev_scalars, lo_slot);
        }
        c.sync();
        const double hi = c.host_scalars[0];
        *result = a->dtype == OWTK_F64 ? hi : static_cast<double>(static_cast<float>(hi));
        if (low != nullptr) *low = a->dtype == OWTK_F64 ? c.host_scalars[1] : 0.0;
    });
}

owtk_status owtk_norm_ex(owtk_vector* a, owtk_reduction_kind reduction, double* result)
{
    return guarded([&] {
        require(a != nullptr && result != nullptr, "null handle");
        if (reduction < OWTK_REDUCTION_SERIAL || reduction > OWTK_REDUCTION_MIXED_PRECISION)
            fail(OWTK_ERR_INVALID_ARGUMENT, "unknown reduction kind");
        if (reduction != OWTK_REDUCTION_MIXED_PRECISION) {   // the compensated norm is the serial one
            const owtk_status st = owtk_norm(a, result);
            if (st != OWTK_OK) fail(st, owtk_last_error());
            return;
        }
        Context& c = *a->ctx;
        double* scratch = c.dev_scalar_copy.as<double>() + 8;
        if (a->dtype == OWTK_F64)
            kern::norm_accurate<double>(c, a->owned_size(), static_cast<const double*>(a->data), scratch,
                                        c.dev_scalar_copy.as<double>(), c.dev_scalars);
        else
            kern::norm_accurate<float>(c, a->owned_size(), static_cast<const float*>(a->data), scratch,
                                       c.dev_scalar_copy.as<double>(), c.dev_scalars);
        c.sync();
        *result = a->dtype == OWTK_F64 ? c.host_scalars[0] : static_cast<double>(static_cast<float>(c.host_scalars[0]));
    });
}

owtk_status owtk_arnoldi_snapshot_create(owtk_context* ctx, owtk_arnoldi_snapshot** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr, "null handle");
        auto s = std::make_unique<owtk_arnoldi_snapshot>();
        s->ctx = ctx;
        *out = s.release();
    });
}

owtk_status owtk_arnoldi_snapshot_destroy(owtk_arnoldi_snapshot* snapshot)
{
    return guarded([&] { delete snapshot; });
}

owtk_status owtk_arnoldi_snapshot_clear(owtk_arnoldi_snapshot* snapshot)
{
    return guarded([&] {
        require(snapshot != nullptr, "null handle");
        snapshot->clear();
    });
}

size_t owtk_arnoldi_snapshot_columns(const owtk_arnoldi_snapshot* snapshot)
{
    return snapshot ? snapshot->columns : 0;
}

owtk_status owtk_arnoldi_snapshot_h(const owtk_arnoldi_snapshot* snapshot, size_t row, size_t column, double* value)
{
    return guarded([&] {
        require(snapshot != nullptr && value != nullptr, "null handle");
        if (column >= snapshot->columns || row > snapshot->columns) fail(OWTK_ERR_OUT_OF_RANGE, "Arnoldi snapshot entry");
        *value = snapshot->h[column * (snapshot->max_columns + 1) + row];
    });
}

owtk_status owtk_arnoldi_snapshot_basis(owtk_arnoldi_snapshot* snapshot, size_t column, owtk_vector** out)
{
    return guarded([&] {
        require(snapshot != nullptr && out != nullptr, "null handle");
        if (column >= snapshot->columns) fail(OWTK_ERR_OUT_OF_RANGE, "Arnoldi snapshot basis");
        snapshot->ctx->sync();
        *out = static_cast<owtk_vector*>(snapshot->basis[column].get());
    });
}

owtk_status owtk_callback_operator_create(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost, size_t bs,
                                          owtk_host_apply_fn apply, void* user, owtk_matrix** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr && apply != nullptr, "null handle");
        if (owned == 0 || bs == 0) fail(OWTK_ERR_INVALID_ARGUMENT, "invalid operator layout");
        if (dtype != OWTK_F64 && dtype != OWTK_F32) fail(OWTK_ERR_INVALID_ARGUMENT, "operator dtype must be F64 or F32");
        auto m = std::make_unique<owtk_matrix>();
        m->ctx = ctx;
        m->kind = 3;
        m->dtype = dtype;
        m->owned = owned;
        m->ghost = ghost;
        m->bs = bs;
        m->host_apply = apply;
        m->host_user = user;
        *out = m.release();
    });
}

owtk_status owtk_pc_create_callback(owtk_context* ctx, owtk_dtype dtype, size_t owned, size_t ghost, size_t bs,
                                    owtk_host_apply_fn apply, void* user, owtk_preconditioner** out)
{
    return guarded([&] {
        require(ctx != nullptr && out != nullptr && apply != nullptr, "null handle");
        if (owned == 0 || bs == 0) fail(OWTK_ERR_INVALID_ARGUMENT, "invalid preconditioner layout");
        if (dtype != OWTK_F64 && dtype != OWTK_F32)
            fail(OWTK_ERR_INVALID_ARGUMENT, "preconditioner dtype must be F64 or F32");
        auto p = std::make_unique<owtk_preconditioner>();
        p->ctx = ctx;
        p->kind = OWTK_PC_CALLBACK;
        p->dtype = dtype;
        p->owned = owned;
        p->ghost = ghost;
        p->bs = bs;
        p->host_apply = apply;
        p->host_user = user;
        *out = p.release();
    });
}

namespace {
SolveExtras extras_of(owtk_solver_kind kind, const owtk_solve_extras* e)
{
    SolveExtras x;
    if (e == nullptr) return x;
    if (e->reduction < OWTK_REDUCTION_SERIAL || e->reduction > OWTK_REDUCTION_MIXED_PRECISION || e->reserved != 0)
        fail(OWTK_ERR_INVALID_ARGUMENT, "unknown reduction kind");
    if (e->arnoldi_snapshot != nullptr && kind != OWTK_SOLVER_FGMRES)
        fail(OWTK_ERR_INVALID_ARGUMENT, "Arnoldi snapshots are recorded by FGMRES only");
    x.reduction = e->reduction;
    x.test = e->convergence_test;
    x.user = e->convergence_user;
    x.snapshot = e->arnoldi_snapshot;
    return x;
}
}  // namespace

owtk_status owtk_solve_ex(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc, owtk_vector* rhs,
                          owtk_vector* x, const owtk_solver_options* options, owtk_workspace* workspace,
                          const owtk_solve_extras* extras, owtk_solver_result* result)
{
    return guarded([&] {
        require(m != nullptr && rhs != nullptr && x != nullptr && options != nullptr && result != nullptr,
                "null handle");
        const SolveExtras ex = extras_of(kind, extras);
        owtk_workspace local;
        local.ctx = m->ctx;
        Workspace& ws = workspace ? static_cast<Workspace&>(*workspace) : static_cast<Workspace&>(local);
        solve(kind, *m, pc, *rhs, *x, *options, ws, *result, &ex);
    });
}

// ------------------------------------------------------------ solves
owtk_status owtk_solve(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc, owtk_vector* rhs,
                       owtk_vector* x, const owtk_solver_options* options, owtk_workspace* workspace,
                       owtk_solver_result* result)
{
    return guarded([&] {
        require(m != nullptr && rhs != nullptr && x != nullptr && options != nullptr && result != nullptr,
                "null handle");
        owtk_workspace local;
        local.ctx = m->ctx;
        Workspace& ws = workspace ? static_cast<Workspace&>(*workspace) : static_cast<Workspace&>(local);
        solve(kind, *m, pc, *rhs, *x, *options, ws, *result);
    });
}

// solve_specwave_native (specwave_compat.hpp:99-249): the legacy SpecWave
// solver IDs mapped onto the device solvers and preconditioners exactly as the
// reference maps them.  ID 10 takes the mixed-precision reduction and ID 22
// the compensated one whatever the caller passes (specwave_compat.hpp:157-176,
// :223-243); the others take the caller's.  Stationary and multigrid IDs are
// not on this path.
owtk_status owtk_solve_specwave(int solver_id, owtk_matrix* m, owtk_vector* rhs, owtk_vector* x,
                                const owtk_solver_options* options, owtk_workspace* workspace,
                                owtk_solver_result* result)
{
    return owtk_solve_specwave_ex(solver_id, m, rhs, x, options, workspace, OWTK_REDUCTION_SERIAL, result);
}

owtk_status owtk_solve_specwave_ex(int solver_id, owtk_matrix* m, owtk_vector* rhs, owtk_vector* x,
                                   const owtk_solver_options* options, owtk_workspace* workspace,
                                   owtk_reduction_kind reduction, owtk_solver_result* result)
{
    return guarded([&] {
        if (reduction < OWTK_REDUCTION_SERIAL || reduction > OWTK_REDUCTION_MIXED_PRECISION)
            fail(OWTK_ERR_INVALID_ARGUMENT, "unknown reduction kind");
        SolveExtras ex;
        ex.reduction = solver_id == 10 ? OWTK_REDUCTION_MIXED_PRECISION
                     : solver_id == 22 ? OWTK_REDUCTION_COMPENSATED : reduction;
        require(m != nullptr && rhs != nullptr && x != nullptr && options != nullptr && result != nullptr,
                "null handle");
        owtk_solver_options o = *options;
        owtk_solver_kind kind = OWTK_SOLVER_BICGSTAB;
        owtk_pc_kind pck = OWTK_PC_SSOR;
        double parameter = o.relaxation;
        switch (solver_id) {
        case 3: case 10: case 22: kind = OWTK_SOLVER_COMM_HIDING_BICGSTAB; break;
        case 4:
            kind = OWTK_SOLVER_COMM_HIDING_BICGSTAB;
            if (o.residual_replacement_interval == 0) o.residual_replacement_interval = 50;
            break;
        case 5: case 8: case 11: kind = OWTK_SOLVER_BICGSTAB; break;
        case 7: kind = OWTK_SOLVER_FGMRES; break;
        case 9: case 13: kind = OWTK_SOLVER_BICGSTAB; pck = OWTK_PC_ILU; parameter = 0; break;
        case 12: case 15: kind = OWTK_SOLVER_PIPELINED_BICGSTAB; break;
        case 14: kind = OWTK_SOLVER_IDRS; break;
        case 21: kind = OWTK_SOLVER_PIPELINED_BICGSTAB; pck = OWTK_PC_ILU; parameter = 0; break;
        case 6: {   // the PETSc adapter: a default SolverResult
            owtk_solver_result r{};
            r.status = 4;
            const double nan = std::numeric_limits<double>::quiet_NaN();
            r.initial_residual_norm = r.recursive_residual_norm = r.true_residual_norm = r.relative_residual_norm = nan;
            *result = r;
            return;
        }
        default:
            fail(OWTK_ERR_INVALID_ARGUMENT, "SpecWave solver id is not on the device path (stationary or multigrid)");
        }
        auto pc = make_pc(m, pck, parameter, OWTK_F64);
        owtk_workspace local;
        local.ctx = m->ctx;
        Workspace& ws = workspace ? static_cast<Workspace&>(*workspace) : static_cast<Workspace&>(local);
        solve(kind, *m, pc.get(), *rhs, *x, o, ws, *result, &ex);
    });
}

owtk_status owtk_solve_host(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc,
                            const void* host_rhs, void* host_x, const owtk_solver_options* options,
                            owtk_workspace* workspace, owtk_solver_result* result)
{
    return owtk_solve_host_ex(kind, m, pc, host_rhs, host_x, options, workspace, nullptr, result);
}

owtk_status owtk_solve_host_ex(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc,
                               const void* host_rhs, void* host_x, const owtk_solver_options* options,
                               owtk_workspace* workspace, const owtk_solve_extras* extras,
                               owtk_solver_result* result)
{
    return guarded([&] {
        require(m != nullptr && host_rhs != nullptr && host_x != nullptr && options != nullptr
                    && result != nullptr,
                "null handle");
        const SolveExtras ex = extras_of(kind, extras);
        Context& c = *m->ctx;
        owtk_workspace local;
        local.ctx = m->ctx;
        Workspace& ws = workspace ? static_cast<Workspace&>(*workspace) : static_cast<Workspace&>(local);
        // The rhs/x staging vectors are kept in the workspace, so repeated
        // calls with the same workspace allocate nothing.
        owtk_vector layout;
        layout.ctx = m->ctx;
        layout.dtype = m->dtype;
        layout.owned = m->owned;
        layout.ghost = m->ghost;
        layout.bs = m->bs;
        auto stage = [&](std::size_t i) -> Vector& {
            if (ws.stage.size() <= i || !ws.stage[i]->same_layout(layout) || ws.stage[i]->dtype != layout.dtype) {
                if (ws.stage.size() <= i) ws.stage.resize(i + 1);
                auto v = std::make_unique<owtk_vector>();
                v->ctx = m->ctx;
                v->dtype = layout.dtype;
                v->owned = layout.owned;
                v->ghost = layout.ghost;
                v->bs = layout.bs;
                v->storage.allocate(layout.local_size() * layout.elem());
                v->data = v->storage.ptr;
                ws.stage[i] = std::move(v);
            }
            return *ws.stage[i];
        };
        Vector& b = stage(0);
        Vector& x = stage(1);
        const std::size_t bytes = layout.local_size() * layout.elem();
        OWTK_CUDA(cudaMemcpyAsync(b.data, host_rhs, bytes, cudaMemcpyHostToDevice, c.stream));
        OWTK_CUDA(cudaMemcpyAsync(x.data, host_x, bytes, cudaMemcpyHostToDevice, c.stream));
        solve(kind, *m, pc, b, x, *options, ws, *result, &ex);
        OWTK_CUDA(cudaMemcpyAsync(host_x, x.data, bytes, cudaMemcpyDeviceToHost, c.stream));
        c.sync();
    });
}

owtk_vector* owtk_workspace_vector(owtk_workspace* ws, size_t index)
{
    if (!ws || index >= ws->vectors.size()) return nullptr;
    return static_cast<owtk_vector*>(ws->vectors[index].get());
}

}  // extern "C"
