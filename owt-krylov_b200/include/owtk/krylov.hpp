// owtk/krylov.hpp — header-only C++20 API of the B200 solve path.
//
// The names, constructors and call signatures of OWT-Krylov's header-only API
// (namespace owt::krylov: BlockVector, BlockCsrMatrix, SplitBlockCsrMatrixView,
// DenseBlockCsrMatrix, PolicyBlockOperator, DistributedBlockOperator, the
// Jacobi / SSOR / split-SSOR / ILU(k) preconditioners, SolverOptions /
// SolverResult / SolverWorkspace and the solver free functions), implemented
// over the C ABI of owtk.h.  A consumer switches by including this header in
// place of the reference's umbrella header and selecting CudaExecutionPolicy
// (the default policy here); solves then run device-resident on the GPU, with
// host vectors copied in and out once per solve.
//
// Differences a consumer must know:
//   * Host coefficient arrays are copied to the device when a matrix is first
//     used; after writing coefficients in place, call sync_values() on the
//     matrix (preconditioner update_values(matrix) does it too).  The
//     reference reads host arrays at every apply instead.
//   * SolverOptions::convergence_test is called with a host copy of each
//     candidate iterate (one device-to-host copy per call).
//   * Reductions run on the device: SerialReduction, CompensatedSerialReduction
//     and MixedPrecisionSerialReduction select the matching device reduction;
//     any other Reduction type reduces like SerialReduction.
//   * Operators and preconditioners that are not this header's types (any
//     type with apply(in, out)) are called on host copies of the vectors once
//     per application.
// Link with -lowtk_b200 and add the repository's include/ directory.
#pragma once

#if defined(__FAST_MATH__) || (defined(__FINITE_MATH_ONLY__) && __FINITE_MATH_ONLY__ > 0)
#error "owtk requires finite-value checks: disable -ffast-math and -ffinite-math-only"
#endif

#include <owtk.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <concepts>
#include <cstddef>
#include <cstdint>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <span>
#include <stdexcept>
#include <string>
#include <string_view>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

namespace owt::krylov {

// ------------------------------------------------------------------ enums
enum class SolverStatus { converged, maximum_iterations, breakdown, diverged, invalid_input };

enum class GmresOrthogonalization {
    iterated_classical_gram_schmidt,
    adaptive_classical_gram_schmidt,
    one_synchronization_classical_gram_schmidt,
};

enum class BreakdownReason {
    none,
    arnoldi_invariant_subspace,
    singular_projected_system,
    biorthogonality_loss,
    alpha_denominator,
    omega_denominator,
    omega_zero,
    idr_shadow_space,
    idr_small_system,
    non_finite_scalar,
};

[[nodiscard]] constexpr std::string_view to_string(BreakdownReason r) noexcept
{
    constexpr std::string_view names[] = {"none", "arnoldi_invariant_subspace", "singular_projected_system",
                                          "biorthogonality_loss", "alpha_denominator", "omega_denominator",
                                          "omega_zero", "idr_shadow_space", "idr_small_system",
                                          "non_finite_scalar"};
    const auto i = static_cast<std::size_t>(r);
    return i < std::size(names) ? names[i] : "unknown";
}

[[nodiscard]] constexpr std::string_view to_string(SolverStatus s) noexcept
{
    constexpr std::string_view names[] = {"converged", "maximum_iterations", "breakdown", "diverged",
                                          "invalid_input"};
    const auto i = static_cast<std::size_t>(s);
    return i < std::size(names) ? names[i] : "unknown";
}

template<std::floating_point T> class BlockVector;

template<std::floating_point T>
struct SolverOptions {
    T relative_tolerance = T(1e-8);
    T absolute_tolerance = T(0);
    T breakdown_tolerance = T(64) * std::numeric_limits<T>::epsilon();
    std::size_t maximum_iterations = 1000;
    std::size_t convergence_check_interval = 10;
    std::size_t restart = 30;
    std::size_t residual_replacement_interval = 50;
    std::size_t idr_shadow_space = 4;
    T relaxation = T(1);
    bool verify_true_residual = true;
    bool collect_timings = false;
    std::function<bool(std::size_t, const BlockVector<T>&)> convergence_test;
    GmresOrthogonalization gmres_orthogonalization = GmresOrthogonalization::iterated_classical_gram_schmidt;
};

template<std::floating_point T>
struct SolverTimings {
    double solve_seconds = 0;
};

template<std::floating_point T>
struct SolverResult {
    SolverStatus status = SolverStatus::invalid_input;
    BreakdownReason breakdown_reason = BreakdownReason::none;
    std::size_t iterations = 0;
    std::size_t operator_applications = 0;
    std::size_t preconditioner_applications = 0;
    std::size_t global_reductions = 0;
    std::size_t reorthogonalizations = 0;
    std::size_t arnoldi_norm_verifications = 0;
    T initial_residual_norm = std::numeric_limits<T>::quiet_NaN();
    T recursive_residual_norm = std::numeric_limits<T>::quiet_NaN();
    T true_residual_norm = std::numeric_limits<T>::quiet_NaN();
    T relative_residual_norm = std::numeric_limits<T>::quiet_NaN();
    bool converged_by_application = false;
    std::shared_ptr<SolverTimings<T>> timings;

    [[nodiscard]] constexpr bool converged() const noexcept { return status == SolverStatus::converged; }
    [[nodiscard]] double solve_seconds() const noexcept { return timings ? timings->solve_seconds : 0; }
};

// ------------------------------------------------------------------ runtime
namespace cuda {

// C ABI status -> the reference's exception types.
[[noreturn]] inline void throw_status(owtk_status s)
{
    const std::string msg = owtk_last_error();
    switch (s) {
    case OWTK_ERR_INVALID_ARGUMENT: throw std::invalid_argument(msg);
    case OWTK_ERR_OUT_OF_RANGE: throw std::out_of_range(msg);
    case OWTK_ERR_ZERO_PIVOT: throw std::runtime_error("zero pivot in ILU(0)");
    default: throw std::runtime_error("owtk: " + msg);
    }
}

inline void check(owtk_status s)
{
    if (s != OWTK_OK) throw_status(s);
}

template<class T> constexpr owtk_dtype dtype_of() { return std::same_as<T, double> ? OWTK_F64 : OWTK_F32; }

// One context (device + stream) per process; device 0 unless OWTK_DEVICE is set.
class Runtime {
public:
    static Runtime& instance()
    {
        static Runtime r;
        return r;
    }
    owtk_context* context()
    {
        std::lock_guard<std::mutex> lock(mutex_);
        if (!ctx_) {
            const char* dev = std::getenv("OWTK_DEVICE");
            owtk_context* c = nullptr;
            check(owtk_context_create(dev ? std::atoi(dev) : 0, &c));
            ctx_.reset(c, [](owtk_context* p) { owtk_context_destroy(p); });
        }
        return ctx_.get();
    }
    // Two device vectors of a layout, reused by host-vector applies.
    std::pair<owtk_vector*, owtk_vector*> scratch(owtk_dtype d, std::size_t owned, std::size_t ghost, std::size_t bs)
    {
        auto* ctx = context();
        std::lock_guard<std::mutex> lock(mutex_);
        auto key = std::make_tuple(static_cast<int>(d), owned, ghost, bs);
        auto it = scratch_.find(key);
        if (it == scratch_.end()) {
            owtk_vector *a = nullptr, *b = nullptr;
            check(owtk_vector_create(ctx, d, owned, ghost, bs, &a));
            check(owtk_vector_create(ctx, d, owned, ghost, bs, &b));
            it = scratch_.emplace(key, std::make_pair(a, b)).first;
        }
        return it->second;
    }
    ~Runtime()
    {
        for (auto& [k, v] : scratch_) {
            owtk_vector_destroy(v.first);
            owtk_vector_destroy(v.second);
        }
    }

private:
    std::mutex mutex_;
    std::shared_ptr<owtk_context> ctx_;
    std::map<std::tuple<int, std::size_t, std::size_t, std::size_t>, std::pair<owtk_vector*, owtk_vector*>> scratch_;
};

template<class H, class D>
std::shared_ptr<H> own(H* h, D d)
{
    return std::shared_ptr<H>(h, d);
}

}  // namespace cuda

// ------------------------------------------------------------------ BlockVector
// Owned nodes first, ghost nodes second, bs contiguous values per node
// (core.hpp:193-395).  Host storage; solves copy it to the device once.
template<std::floating_point T>
class BlockVector {
public:
    using value_type = T;
    BlockVector() = default;
    BlockVector(std::size_t owned_nodes, std::size_t ghost_nodes, std::size_t block_size, T initial_value = T(0))
        : owned_(owned_nodes), ghost_(ghost_nodes), bs_(block_size),
          storage_((owned_nodes + ghost_nodes) * block_size, initial_value)
    {
        validate(storage_.size());
        values_ = storage_;
    }
    [[nodiscard]] static BlockVector view(std::size_t owned_nodes, std::size_t ghost_nodes, std::size_t block_size,
                                          std::span<T> values)
    {
        BlockVector v;
        v.owned_ = owned_nodes;
        v.ghost_ = ghost_nodes;
        v.bs_ = block_size;
        v.validate(values.size());
        v.values_ = values;
        v.is_view_ = true;
        return v;
    }
    BlockVector(const BlockVector& o) : owned_(o.owned_), ghost_(o.ghost_), bs_(o.bs_), is_view_(o.is_view_)
    {
        if (is_view_) values_ = o.values_;
        else { storage_.assign(o.values_.begin(), o.values_.end()); values_ = storage_; }
    }
    BlockVector& operator=(const BlockVector& o)
    {
        if (this == &o) return *this;
        owned_ = o.owned_; ghost_ = o.ghost_; bs_ = o.bs_; is_view_ = o.is_view_;
        if (is_view_) { storage_.clear(); values_ = o.values_; }
        else { storage_.assign(o.values_.begin(), o.values_.end()); values_ = storage_; }
        return *this;
    }
    BlockVector(BlockVector&& o) noexcept
        : owned_(o.owned_), ghost_(o.ghost_), bs_(o.bs_), storage_(std::move(o.storage_)), is_view_(o.is_view_)
    {
        values_ = is_view_ ? o.values_ : std::span<T>(storage_);
        o.reset();
    }
    BlockVector& operator=(BlockVector&& o) noexcept
    {
        if (this == &o) return *this;
        owned_ = o.owned_; ghost_ = o.ghost_; bs_ = o.bs_;
        storage_ = std::move(o.storage_);
        is_view_ = o.is_view_;
        values_ = is_view_ ? o.values_ : std::span<T>(storage_);
        o.reset();
        return *this;
    }

    [[nodiscard]] std::size_t owned_nodes() const noexcept { return owned_; }
    [[nodiscard]] std::size_t ghost_nodes() const noexcept { return ghost_; }
    [[nodiscard]] std::size_t local_nodes() const noexcept { return owned_ + ghost_; }
    [[nodiscard]] std::size_t block_size() const noexcept { return bs_; }
    [[nodiscard]] std::size_t owned_size() const noexcept { return owned_ * bs_; }
    [[nodiscard]] std::size_t local_size() const noexcept { return values_.size(); }
    [[nodiscard]] bool owns_memory() const noexcept { return !is_view_; }
    [[nodiscard]] T* data() noexcept { return values_.data(); }
    [[nodiscard]] const T* data() const noexcept { return values_.data(); }
    [[nodiscard]] std::span<T> owned() noexcept { return {values_.data(), owned_size()}; }
    [[nodiscard]] std::span<const T> owned() const noexcept { return {values_.data(), owned_size()}; }
    [[nodiscard]] std::span<T> ghosts() noexcept { return {values_.data() + owned_size(), ghost_ * bs_}; }
    [[nodiscard]] std::span<const T> ghosts() const noexcept { return {values_.data() + owned_size(), ghost_ * bs_}; }
    [[nodiscard]] std::span<T> node(std::size_t i)
    {
        if (i >= local_nodes()) throw std::out_of_range("BlockVector node index");
        return {values_.data() + i * bs_, bs_};
    }
    [[nodiscard]] std::span<const T> node(std::size_t i) const
    {
        if (i >= local_nodes()) throw std::out_of_range("BlockVector node index");
        return {values_.data() + i * bs_, bs_};
    }
    void fill_owned(T v) { std::fill(owned().begin(), owned().end(), v); }
    void fill(T v) { std::fill(values_.begin(), values_.end(), v); }
    [[nodiscard]] BlockVector clone_layout(T v = T(0)) const { return BlockVector(owned_, ghost_, bs_, v); }
    [[nodiscard]] bool same_layout(const BlockVector& o) const noexcept
    {
        return owned_ == o.owned_ && ghost_ == o.ghost_ && bs_ == o.bs_;
    }

private:
    void validate(std::size_t count) const
    {
        if (owned_ == 0 || bs_ == 0 || count != (owned_ + ghost_) * bs_)
            throw std::invalid_argument("invalid BlockVector layout or storage size");
    }
    void reset() noexcept
    {
        owned_ = ghost_ = bs_ = 0;
        storage_.clear();
        values_ = {};
        is_view_ = false;
    }
    std::size_t owned_ = 0, ghost_ = 0, bs_ = 0;
    std::vector<T> storage_;
    std::span<T> values_;
    bool is_view_ = false;
};

// ------------------------------------------------------------------ workspace
// Device vectors reused across solves of one layout (core.hpp:397-459).
template<std::floating_point T>
class SolverWorkspace {
public:
    [[nodiscard]] std::size_t allocation_epochs() const noexcept
    {
        return ws_ ? static_cast<std::size_t>(owtk_workspace_allocation_epochs(ws_.get())) : 0;
    }
    owtk_workspace* handle()
    {
        if (!ws_) {
            owtk_workspace* w = nullptr;
            cuda::check(owtk_workspace_create(cuda::Runtime::instance().context(), &w));
            ws_ = cuda::own(w, [](owtk_workspace* p) { owtk_workspace_destroy(p); });
        }
        return ws_.get();
    }
    // Copy of workspace vector `index` (the reference's slot order).
    [[nodiscard]] std::vector<T> vector_values(std::size_t index, std::size_t count)
    {
        owtk_vector* v = owtk_workspace_vector(handle(), index);
        if (!v) throw std::out_of_range("solver workspace vector index");
        std::vector<T> out(count);
        cuda::check(owtk_vector_download(v, out.data(), count));
        return out;
    }

private:
    std::shared_ptr<owtk_workspace> ws_;
};

// ------------------------------------------------------------------ execution
// The device execution policy: the only policy of this header.
struct CudaExecutionPolicy {
    [[nodiscard]] static constexpr const char* name() noexcept { return "cuda-sm100a"; }
    [[nodiscard]] static bool accelerator_available() noexcept
    {
        owtk_context* c = nullptr;
        if (owtk_context_create(0, &c) != OWTK_OK) return false;
        owtk_context_destroy(c);
        return true;
    }
};

namespace detail {

template<class Index>
std::vector<std::uint64_t> widen(std::span<const Index> s)
{
    std::vector<std::uint64_t> out(s.size());
    for (std::size_t i = 0; i < s.size(); ++i) {
        if constexpr (std::signed_integral<Index>)
            if (s[i] < 0) throw std::invalid_argument("negative matrix index");
        out[i] = static_cast<std::uint64_t>(s[i]);
    }
    return out;
}

// Host vectors through a device apply: upload in, run, download owned out.
template<class T, class F>
void apply_host(const BlockVector<T>& in, BlockVector<T>& out, F&& run)
{
    auto [din, dout] = cuda::Runtime::instance().scratch(cuda::dtype_of<T>(), in.owned_nodes(), in.ghost_nodes(),
                                                        in.block_size());
    cuda::check(owtk_vector_upload(din, in.data(), in.local_size()));
    cuda::check(owtk_vector_upload(dout, out.data(), out.local_size()));
    run(din, dout);
    cuda::check(owtk_context_synchronize(cuda::Runtime::instance().context()));
    cuda::check(owtk_vector_download(dout, out.data(), out.owned_size()));
}

}  // namespace detail

// ------------------------------------------------------------------ matrices
// Component-diagonal block CSR, values [entry][component] (block_csr.hpp:17-360).
template<std::floating_point T, std::integral Index = std::size_t>
class BlockCsrMatrix {
public:
    BlockCsrMatrix() = default;
    BlockCsrMatrix(std::size_t owned_nodes, std::size_t ghost_nodes, std::size_t block_size,
                   std::vector<Index> row_offsets, std::vector<Index> column_indices, std::vector<T> values)
        : owned_(owned_nodes), ghost_(ghost_nodes), bs_(block_size), rp_store_(std::move(row_offsets)),
          ci_store_(std::move(column_indices)), v_store_(std::move(values))
    {
        rp_ = rp_store_;
        ci_ = ci_store_;
        v_ = v_store_;
        create();
    }
    [[nodiscard]] static BlockCsrMatrix view(std::size_t owned_nodes, std::size_t ghost_nodes, std::size_t block_size,
                                             std::span<const Index> row_offsets, std::span<const Index> column_indices,
                                             std::span<T> values)
    {
        BlockCsrMatrix m;
        m.owned_ = owned_nodes;
        m.ghost_ = ghost_nodes;
        m.bs_ = block_size;
        m.rp_ = row_offsets;
        m.ci_ = column_indices;
        m.v_ = values;
        m.view_ = true;
        m.create();
        return m;
    }
    BlockCsrMatrix(const BlockCsrMatrix&) = delete;
    BlockCsrMatrix& operator=(const BlockCsrMatrix&) = delete;
    BlockCsrMatrix(BlockCsrMatrix&&) noexcept = default;
    BlockCsrMatrix& operator=(BlockCsrMatrix&&) noexcept = default;

    [[nodiscard]] std::size_t owned_nodes() const noexcept { return owned_; }
    [[nodiscard]] std::size_t ghost_nodes() const noexcept { return ghost_; }
    [[nodiscard]] std::size_t local_nodes() const noexcept { return owned_ + ghost_; }
    [[nodiscard]] std::size_t block_size() const noexcept { return bs_; }
    [[nodiscard]] std::size_t entries() const noexcept { return ci_.size(); }
    [[nodiscard]] bool owns_memory() const noexcept { return !view_; }
    [[nodiscard]] std::span<const Index> row_offsets() const noexcept { return rp_; }
    [[nodiscard]] std::span<const Index> column_indices() const noexcept { return ci_; }
    [[nodiscard]] std::span<const T> values() const noexcept { return v_; }
    [[nodiscard]] std::span<T> values() noexcept { return v_; }

    // Copy the host coefficients to the device after writing them in place.
    void sync_values() { cuda::check(owtk_bsr_update_values(dev_.get(), v_.data())); }
    [[nodiscard]] owtk_matrix* device() const { return dev_.get(); }

    void apply(const BlockVector<T>& in, BlockVector<T>& out) const
    {
        check_vectors(in, out);
        detail::apply_host(in, out, [&](owtk_vector* a, owtk_vector* b) { cuda::check(owtk_spmv(dev_.get(), a, b)); });
    }
    // The listed rows only, as apply computes them; other rows untouched.
    void apply_rows(const BlockVector<T>& in, BlockVector<T>& out, std::span<const std::size_t> rows) const
    {
        check_vectors(in, out);
        const std::vector<std::uint64_t> r(rows.begin(), rows.end());
        detail::apply_host(in, out, [&](owtk_vector* a, owtk_vector* b) {
            cuda::check(owtk_spmv_rows(dev_.get(), a, b, r.data(), r.size()));
        });
    }
    [[nodiscard]] std::vector<T> diagonal() const
    {
        std::vector<T> d(owned_ * bs_);
        cuda::check(owtk_matrix_diagonal(dev_.get(), d.data()));
        return d;
    }

private:
    void create()
    {
        if (owned_ == 0 || bs_ == 0 || rp_.size() != owned_ + 1 || v_.size() != ci_.size() * bs_
            || rp_.empty() || static_cast<std::size_t>(rp_.back()) != ci_.size())
            throw std::invalid_argument("invalid BlockCsrMatrix storage");
        const auto rp = detail::widen<Index>(rp_);
        auto ci = detail::widen<Index>(ci_);
        if (ci.empty()) ci.push_back(0);
        owtk_matrix* m = nullptr;
        cuda::check(owtk_bsr_create(cuda::Runtime::instance().context(), cuda::dtype_of<T>(), owned_, ghost_, bs_,
                                    rp.data(), ci.data(), v_.data(), &m));
        dev_ = cuda::own(m, [](owtk_matrix* p) { owtk_matrix_destroy(p); });
    }
    void check_vectors(const BlockVector<T>& in, const BlockVector<T>& out) const
    {
        if (!in.same_layout(out) || in.owned_nodes() != owned_ || in.ghost_nodes() != ghost_ || in.block_size() != bs_)
            throw std::invalid_argument("BlockCsrMatrix vector layout mismatch");
    }
    std::size_t owned_ = 0, ghost_ = 0, bs_ = 0;
    std::vector<Index> rp_store_, ci_store_;
    std::vector<T> v_store_;
    std::span<const Index> rp_, ci_;
    std::span<T> v_;
    bool view_ = false;
    std::shared_ptr<owtk_matrix> dev_;
};

// Borrowed split diagonal/edge operator (split_block_csr.hpp:17-196).  The
// structure is copied once; the borrowed host coefficients are mirrored in
// device buffers refreshed by sync_values().
template<std::floating_point T, std::integral Index = std::size_t>
class SplitBlockCsrMatrixView {
public:
    SplitBlockCsrMatrixView(std::size_t owned_nodes, std::size_t ghost_nodes, std::size_t block_size,
                            std::span<const Index> off_diagonal_row_offsets, std::span<const Index> off_diagonal_columns,
                            std::span<const T> diagonal, std::span<const T> off_diagonal)
        : owned_(owned_nodes), ghost_(ghost_nodes), bs_(block_size), rp_(off_diagonal_row_offsets),
          ci_(off_diagonal_columns), diag_(diagonal), off_(off_diagonal)
    {
        if (owned_ == 0 || bs_ == 0 || rp_.size() != owned_ + 1 || diag_.size() != owned_ * bs_
            || off_.size() != ci_.size() * bs_)
            throw std::invalid_argument("invalid split CSR storage");
        auto* ctx = cuda::Runtime::instance().context();
        owtk_vector *d = nullptr, *o = nullptr;
        cuda::check(owtk_vector_create(ctx, cuda::dtype_of<T>(), owned_ * bs_, 0, 1, &d));
        cuda::check(owtk_vector_create(ctx, cuda::dtype_of<T>(), std::max<std::size_t>(off_.size(), 1), 0, 1, &o));
        ddiag_ = cuda::own(d, [](owtk_vector* p) { owtk_vector_destroy(p); });
        doff_ = cuda::own(o, [](owtk_vector* p) { owtk_vector_destroy(p); });
        sync_values();
        const auto rp = detail::widen<Index>(rp_);
        auto ci = detail::widen<Index>(ci_);
        if (ci.empty()) ci.push_back(0);
        owtk_matrix* m = nullptr;
        cuda::check(owtk_split_view_create(ctx, cuda::dtype_of<T>(), owned_, ghost_, bs_, rp.data(), ci.data(),
                                           owtk_vector_data(d), owtk_vector_data(o), &m));
        dev_ = cuda::own(m, [](owtk_matrix* p) { owtk_matrix_destroy(p); });
    }
    [[nodiscard]] std::size_t owned_nodes() const noexcept { return owned_; }
    [[nodiscard]] std::size_t ghost_nodes() const noexcept { return ghost_; }
    [[nodiscard]] std::size_t local_nodes() const noexcept { return owned_ + ghost_; }
    [[nodiscard]] std::size_t block_size() const noexcept { return bs_; }
    [[nodiscard]] std::size_t entries() const noexcept { return owned_ + ci_.size(); }
    [[nodiscard]] bool owns_memory() const noexcept { return false; }
    [[nodiscard]] std::span<const Index> off_diagonal_row_offsets() const noexcept { return rp_; }
    [[nodiscard]] std::span<const Index> off_diagonal_columns() const noexcept { return ci_; }
    [[nodiscard]] std::span<const T> diagonal_values() const noexcept { return diag_; }
    [[nodiscard]] std::span<const T> off_diagonal_values() const noexcept { return off_; }
    void sync_values() const
    {
        cuda::check(owtk_vector_upload(ddiag_.get(), diag_.data(), diag_.size()));
        if (!off_.empty()) cuda::check(owtk_vector_upload(doff_.get(), off_.data(), off_.size()));
    }
    [[nodiscard]] owtk_matrix* device() const { return dev_.get(); }
    void apply(const BlockVector<T>& in, BlockVector<T>& out) const
    {
        if (!in.same_layout(out) || in.owned_nodes() != owned_ || in.ghost_nodes() != ghost_ || in.block_size() != bs_)
            throw std::invalid_argument("SplitBlockCsrMatrixView vector layout mismatch");
        detail::apply_host(in, out, [&](owtk_vector* a, owtk_vector* b) { cuda::check(owtk_spmv(dev_.get(), a, b)); });
    }
    // The listed rows only, as apply computes them; other rows untouched.
    void apply_rows(const BlockVector<T>& in, BlockVector<T>& out, std::span<const std::size_t> rows) const
    {
        check_vectors(in, out);
        const std::vector<std::uint64_t> r(rows.begin(), rows.end());
        detail::apply_host(in, out, [&](owtk_vector* a, owtk_vector* b) {
            cuda::check(owtk_spmv_rows(dev_.get(), a, b, r.data(), r.size()));
        });
    }
    [[nodiscard]] std::vector<T> diagonal() const { return {diag_.begin(), diag_.end()}; }

private:
    std::size_t owned_, ghost_, bs_;
    std::span<const Index> rp_, ci_;
    std::span<const T> diag_, off_;
    std::shared_ptr<owtk_vector> ddiag_, doff_;
    std::shared_ptr<owtk_matrix> dev_;
};

// Dense bs x bs block CSR, row-major blocks (dense_block_csr.hpp:15-330).
template<std::floating_point T, std::integral Index = std::size_t>
class DenseBlockCsrMatrix {
public:
    DenseBlockCsrMatrix(std::size_t owned_nodes, std::size_t ghost_nodes, std::size_t block_size,
                        std::vector<Index> row_offsets, std::vector<Index> column_indices, std::vector<T> values)
        : owned_(owned_nodes), ghost_(ghost_nodes), bs_(block_size), rp_(std::move(row_offsets)),
          ci_(std::move(column_indices)), v_(std::move(values))
    {
        if (owned_ == 0 || bs_ == 0 || rp_.size() != owned_ + 1 || v_.size() != ci_.size() * bs_ * bs_)
            throw std::invalid_argument("invalid dense-block CSR storage");
        const auto rp = detail::widen<Index>(std::span<const Index>(rp_));
        auto ci = detail::widen<Index>(std::span<const Index>(ci_));
        if (ci.empty()) ci.push_back(0);
        owtk_matrix* m = nullptr;
        cuda::check(owtk_dense_bsr_create(cuda::Runtime::instance().context(), cuda::dtype_of<T>(), owned_, ghost_, bs_,
                                          rp.data(), ci.data(), v_.data(), &m));
        dev_ = cuda::own(m, [](owtk_matrix* p) { owtk_matrix_destroy(p); });
    }
    [[nodiscard]] std::size_t owned_nodes() const noexcept { return owned_; }
    [[nodiscard]] std::size_t ghost_nodes() const noexcept { return ghost_; }
    [[nodiscard]] std::size_t block_size() const noexcept { return bs_; }
    [[nodiscard]] std::size_t entries() const noexcept { return ci_.size(); }
    [[nodiscard]] std::span<T> values() noexcept { return v_; }
    void sync_values() { cuda::check(owtk_bsr_update_values(dev_.get(), v_.data())); }
    [[nodiscard]] owtk_matrix* device() const { return dev_.get(); }
    void apply(const BlockVector<T>& in, BlockVector<T>& out) const
    {
        if (!in.same_layout(out) || in.owned_nodes() != owned_ || in.ghost_nodes() != ghost_ || in.block_size() != bs_)
            throw std::invalid_argument("dense-block CSR vector layout mismatch");
        detail::apply_host(in, out, [&](owtk_vector* a, owtk_vector* b) { cuda::check(owtk_spmv(dev_.get(), a, b)); });
    }
    // The listed rows only, as apply computes them; other rows untouched.
    void apply_rows(const BlockVector<T>& in, BlockVector<T>& out, std::span<const std::size_t> rows) const
    {
        check_vectors(in, out);
        const std::vector<std::uint64_t> r(rows.begin(), rows.end());
        detail::apply_host(in, out, [&](owtk_vector* a, owtk_vector* b) {
            cuda::check(owtk_spmv_rows(dev_.get(), a, b, r.data(), r.size()));
        });
    }

private:
    std::size_t owned_, ghost_, bs_;
    std::vector<Index> rp_, ci_;
    std::vector<T> v_;
    std::shared_ptr<owtk_matrix> dev_;
};

// ------------------------------------------------------------------ operators
struct NoHaloExchange {
    struct Handle {};
    template<std::floating_point T> void exchange(BlockVector<T>&) const noexcept {}
    template<std::floating_point T> [[nodiscard]] Handle begin(BlockVector<T>&) const noexcept { return {}; }
    void end(Handle&) const noexcept {}
};

// Matrix/halo operator with the kernel selected by policy (execution.hpp:161-195).
template<class Matrix, class ExecutionPolicy = CudaExecutionPolicy, class Halo = NoHaloExchange>
class PolicyBlockOperator {
    static_assert(std::same_as<ExecutionPolicy, CudaExecutionPolicy>,
                  "this header implements the device policy only");

public:
    PolicyBlockOperator(Matrix& matrix, ExecutionPolicy execution = {}, Halo halo = {})
        : matrix_(&matrix), execution_(std::move(execution)), halo_(std::move(halo))
    {
    }
    template<std::floating_point T>
    void apply(BlockVector<T>& input, BlockVector<T>& output)
    {
        halo_.exchange(input);
        matrix_->apply(input, output);
    }
    [[nodiscard]] ExecutionPolicy& execution_policy() noexcept { return execution_; }
    [[nodiscard]] Matrix& matrix() noexcept { return *matrix_; }
    [[nodiscard]] const Matrix& matrix() const noexcept { return *matrix_; }

private:
    Matrix* matrix_;
    ExecutionPolicy execution_;
    Halo halo_;
};

template<class Matrix, class ExecutionPolicy>
PolicyBlockOperator(Matrix&, ExecutionPolicy) -> PolicyBlockOperator<Matrix, ExecutionPolicy>;

// Halo then matrix apply (block_csr.hpp:379-410); on one GPU the halo is empty.
template<class Matrix, class Halo = NoHaloExchange>
class DistributedBlockOperator {
public:
    DistributedBlockOperator(Matrix& matrix, Halo halo = {}) : matrix_(&matrix), halo_(std::move(halo)) {}
    template<std::floating_point T>
    void apply(BlockVector<T>& input, BlockVector<T>& output)
    {
        halo_.exchange(input);
        matrix_->apply(input, output);
    }
    [[nodiscard]] Matrix& matrix() noexcept { return *matrix_; }
    [[nodiscard]] const Matrix& matrix() const noexcept { return *matrix_; }
    [[nodiscard]] Halo& halo() noexcept { return halo_; }

private:
    Matrix* matrix_;
    Halo halo_;
};

template<class Matrix>
DistributedBlockOperator(Matrix&) -> DistributedBlockOperator<Matrix>;

// ------------------------------------------------------------------ preconditioners
struct IdentityPreconditioner {
    template<std::floating_point T>
    void apply(const BlockVector<T>& input, BlockVector<T>& output) const
    {
        if (!input.same_layout(output)) throw std::invalid_argument("BlockVector layout mismatch");
        std::copy(input.owned().begin(), input.owned().end(), output.owned().begin());
    }
    [[nodiscard]] owtk_preconditioner* device() const noexcept { return nullptr; }
};

namespace detail {
// Shared device-preconditioner plumbing.
class DevicePc {
public:
    [[nodiscard]] owtk_preconditioner* device() const noexcept { return pc_.get(); }
    [[nodiscard]] std::size_t numeric_updates() const noexcept
    {
        return static_cast<std::size_t>(owtk_pc_numeric_updates(pc_.get()));
    }
    template<std::floating_point T>
    void apply(const BlockVector<T>& input, BlockVector<T>& output) const
    {
        if (!input.same_layout(output)) throw std::invalid_argument("preconditioner layout mismatch");
        apply_host(input, output, [&](owtk_vector* a, owtk_vector* b) { cuda::check(owtk_pc_apply(pc_.get(), a, b)); });
    }

protected:
    void create(owtk_matrix* m, owtk_pc_kind kind, double parameter)
    {
        owtk_preconditioner* p = nullptr;
        cuda::check(owtk_pc_create(m, kind, parameter, &p));
        pc_ = cuda::own(p, [](owtk_preconditioner* q) { owtk_pc_destroy(q); });
    }
    void refresh(owtk_matrix* m) { cuda::check(owtk_pc_update_values(pc_.get(), m)); }
    std::shared_ptr<owtk_preconditioner> pc_;
};
}  // namespace detail

template<std::floating_point T>
class JacobiPreconditioner : public detail::DevicePc {
public:
    template<class Matrix>
    explicit JacobiPreconditioner(const Matrix& matrix, T minimum_diagonal = T(64) * std::numeric_limits<T>::epsilon())
    {
        create(matrix.device(), OWTK_PC_JACOBI, static_cast<double>(minimum_diagonal));
    }
    template<class Matrix>
    void update_values(Matrix& matrix)
    {
        matrix.sync_values();
        refresh(matrix.device());
    }
};

template<std::floating_point T, std::integral Index>
JacobiPreconditioner(const BlockCsrMatrix<T, Index>&) -> JacobiPreconditioner<T>;
template<std::floating_point T, std::integral Index>
JacobiPreconditioner(const SplitBlockCsrMatrixView<T, Index>&) -> JacobiPreconditioner<T>;

template<std::floating_point T, std::integral Index = std::size_t>
class LocalSsorPreconditioner : public detail::DevicePc {
public:
    // The reference keeps a pointer to the (const) matrix; update_values()
    // re-reads its host values.
    explicit LocalSsorPreconditioner(const BlockCsrMatrix<T, Index>& matrix, T omega = T(1))
        : matrix_(const_cast<BlockCsrMatrix<T, Index>*>(&matrix))
    {
        create(matrix.device(), OWTK_PC_SSOR, static_cast<double>(omega));
    }
    // Refresh the diagonal cache after modifying the referenced matrix.
    void update_values()
    {
        matrix_->sync_values();
        refresh(matrix_->device());
    }

private:
    BlockCsrMatrix<T, Index>* matrix_;
};

template<std::floating_point T, std::integral Index = std::size_t>
class SplitLocalSsorPreconditioner : public detail::DevicePc {
public:
    explicit SplitLocalSsorPreconditioner(const SplitBlockCsrMatrixView<T, Index>& matrix, T omega = T(1))
    {
        create(matrix.device(), OWTK_PC_SPLIT_SSOR, static_cast<double>(omega));
    }
    void update_values(const SplitBlockCsrMatrixView<T, Index>& matrix)
    {
        matrix.sync_values();
        refresh(matrix.device());
    }
};

template<std::floating_point T, std::integral Index = std::size_t>
class IluLevelPreconditioner : public detail::DevicePc {
public:
    explicit IluLevelPreconditioner(const BlockCsrMatrix<T, Index>& matrix, std::size_t fill_level = 0)
        : fill_(fill_level), owned_(matrix.owned_nodes()), bs_(matrix.block_size())
    {
        create(matrix.device(), OWTK_PC_ILU, static_cast<double>(fill_level));
    }
    void update_values(BlockCsrMatrix<T, Index>& matrix)
    {
        matrix.sync_values();
        refresh(matrix.device());
    }
    [[nodiscard]] std::size_t fill_level() const noexcept { return fill_; }
    // Factor storage copied back from the device (preconditioner.hpp:365-370).
    [[nodiscard]] std::vector<std::size_t> factor_row_offsets() const { return factors().rp; }
    [[nodiscard]] std::vector<std::size_t> factor_columns() const { return factors().ci; }
    [[nodiscard]] std::vector<T> factor_values() const { return factors().v; }
    [[nodiscard]] std::vector<T> inverse_diagonal() const { return factors().inv; }

private:
    struct Factors {
        std::vector<std::size_t> rp, ci;
        std::vector<T> v, inv;
    };
    Factors factors() const
    {
        std::uint64_t n = 0;
        cuda::check(owtk_ilu_factors(pc_.get(), &n, nullptr, nullptr, nullptr, nullptr));
        std::vector<std::uint64_t> rp(owned_ + 1), ci(std::max<std::uint64_t>(n, 1));
        Factors f;
        f.v.resize(n * bs_);
        f.inv.resize(owned_ * bs_);
        cuda::check(owtk_ilu_factors(pc_.get(), &n, rp.data(), ci.data(), f.v.data(), f.inv.data()));
        f.rp.assign(rp.begin(), rp.end());
        f.ci.assign(ci.begin(), ci.begin() + static_cast<std::ptrdiff_t>(n));
        return f;
    }
    std::size_t fill_, owned_, bs_;
};

template<std::floating_point T, std::integral Index = std::size_t>
class Ilu0Preconditioner : public IluLevelPreconditioner<T, Index> {
public:
    explicit Ilu0Preconditioner(const BlockCsrMatrix<T, Index>& matrix) : IluLevelPreconditioner<T, Index>(matrix, 0) {}
};

// ------------------------------------------------------------------ reductions
// Device reductions of host vectors (reduction.hpp:103-299).  Solvers given
// one of these three types run their reductions on the device with the same
// accuracy class: serial (two-stage FP64 sums), compensated (Neumaier pairs)
// or mixed precision (doubled-precision Dot2 sums and norm).  Any other
// Reduction type is accepted for source compatibility and reduces serially.
namespace detail {

template<std::floating_point T>
std::pair<double, double> device_dot(const BlockVector<T>& a, const BlockVector<T>& b, owtk_reduction_kind kind)
{
    if (!a.same_layout(b)) throw std::invalid_argument("dot layout mismatch");
    auto [da, db] = cuda::Runtime::instance().scratch(cuda::dtype_of<T>(), a.owned_nodes(), a.ghost_nodes(),
                                                      a.block_size());
    cuda::check(owtk_vector_upload(da, a.data(), a.owned_size()));
    cuda::check(owtk_vector_upload(db, b.data(), b.owned_size()));
    double hi = 0, lo = 0;
    cuda::check(owtk_dot_ex(da, db, kind, &hi, &lo));
    return {hi, lo};
}

template<std::floating_point T>
T device_norm(const BlockVector<T>& a, owtk_reduction_kind kind)
{
    auto [da, db] = cuda::Runtime::instance().scratch(cuda::dtype_of<T>(), a.owned_nodes(), a.ghost_nodes(),
                                                      a.block_size());
    (void)db;
    cuda::check(owtk_vector_upload(da, a.data(), a.owned_size()));
    double r = 0;
    cuda::check(owtk_norm_ex(da, kind, &r));
    return static_cast<T>(r);
}

template<std::floating_point T, owtk_reduction_kind Kind>
class DeviceReduction {
public:
    struct Request {};
    static constexpr owtk_reduction_kind device_kind = Kind;

    [[nodiscard]] T dot(const BlockVector<T>& lhs, const BlockVector<T>& rhs) const
    {
        return static_cast<T>(device_dot(lhs, rhs, Kind).first);
    }
    [[nodiscard]] T local_dot(const BlockVector<T>& lhs, const BlockVector<T>& rhs) const { return dot(lhs, rhs); }
    [[nodiscard]] T norm(const BlockVector<T>& vector) const { return device_norm(vector, Kind); }
    void sum(std::span<const T> local, std::span<T> global) const
    {
        if (local.size() != global.size()) throw std::invalid_argument("reduction batch size mismatch");
        std::copy(local.begin(), local.end(), global.begin());
    }
    [[nodiscard]] Request begin_sum(std::span<const T> local, std::span<T> global) const
    {
        sum(local, global);
        return {};
    }
    void end(Request&) const noexcept {}
};

template<class R>
constexpr owtk_reduction_kind reduction_kind_of()
{
    if constexpr (requires { R::device_kind; }) return R::device_kind;
    else return OWTK_REDUCTION_SERIAL;
}

}  // namespace detail

template<std::floating_point T>
class SerialReduction : public detail::DeviceReduction<T, OWTK_REDUCTION_SERIAL> {};

// Neumaier-compensated reduction (reduction.hpp:175-226).
template<std::floating_point T>
class CompensatedSerialReduction : public detail::DeviceReduction<T, OWTK_REDUCTION_COMPENSATED> {};

// Wide local products (reduction.hpp:228-299): local_dot returns long double,
// here the device's doubled-precision (sum, correction) pair added in long double.
template<std::floating_point T>
class MixedPrecisionSerialReduction {
public:
    struct Request {};
    static constexpr owtk_reduction_kind device_kind = OWTK_REDUCTION_MIXED_PRECISION;

    [[nodiscard]] T dot(const BlockVector<T>& lhs, const BlockVector<T>& rhs) const
    {
        return static_cast<T>(local_dot(lhs, rhs));
    }
    [[nodiscard]] long double local_dot(const BlockVector<T>& lhs, const BlockVector<T>& rhs) const
    {
        const auto [hi, lo] = detail::device_dot(lhs, rhs, device_kind);
        return static_cast<long double>(hi) + static_cast<long double>(lo);
    }
    [[nodiscard]] T norm(const BlockVector<T>& vector) const { return detail::device_norm(vector, device_kind); }
    void sum(std::span<const long double> local, std::span<T> global) const
        requires(!std::same_as<T, long double>)
    {
        if (local.size() != global.size()) throw std::invalid_argument("reduction batch size mismatch");
        std::transform(local.begin(), local.end(), global.begin(), [](long double v) { return static_cast<T>(v); });
    }
    [[nodiscard]] Request begin_sum(std::span<const long double> local, std::span<T> global) const
        requires(!std::same_as<T, long double>)
    {
        sum(local, global);
        return {};
    }
    void sum(std::span<const T> local, std::span<T> global) const
    {
        if (local.size() != global.size()) throw std::invalid_argument("reduction batch size mismatch");
        std::copy(local.begin(), local.end(), global.begin());
    }
    [[nodiscard]] Request begin_sum(std::span<const T> local, std::span<T> global) const
    {
        sum(local, global);
        return {};
    }
    void end(Request&) const noexcept {}
};

// ------------------------------------------------------------------ Arnoldi snapshot
// The last unrotated Arnoldi relation produced by FGMRES (core.hpp:462-534),
// recorded on the device; preconditioned_basis() copies a vector to the host
// on first access after a solve.
template<std::floating_point T>
class ArnoldiSnapshot {
public:
    void clear() noexcept
    {
        if (s_) owtk_arnoldi_snapshot_clear(s_.get());
        cache_.clear();
    }
    [[nodiscard]] std::size_t columns() const noexcept { return s_ ? owtk_arnoldi_snapshot_columns(s_.get()) : 0; }
    [[nodiscard]] T h(std::size_t row, std::size_t column) const
    {
        if (!s_) throw std::out_of_range("Arnoldi snapshot entry");
        double v = 0;
        cuda::check(owtk_arnoldi_snapshot_h(s_.get(), row, column, &v));
        return static_cast<T>(v);
    }
    [[nodiscard]] const BlockVector<T>& preconditioned_basis(std::size_t column) const
    {
        if (!s_ || column >= columns()) throw std::out_of_range("Arnoldi snapshot basis");
        if (cache_.size() != columns()) cache_.assign(columns(), BlockVector<T>());
        if (cache_[column].owned_nodes() == 0) {
            owtk_vector* v = nullptr;
            cuda::check(owtk_arnoldi_snapshot_basis(s_.get(), column, &v));
            BlockVector<T> host(owned_, ghost_, bs_);
            cuda::check(owtk_vector_download(v, host.data(), host.owned_size()));
            cache_[column] = std::move(host);
        }
        return cache_[column];
    }
    // The device snapshot a solve records into (created on first use).
    owtk_arnoldi_snapshot* device_for(std::size_t owned, std::size_t ghost, std::size_t bs)
    {
        if (!s_) {
            owtk_arnoldi_snapshot* p = nullptr;
            cuda::check(owtk_arnoldi_snapshot_create(cuda::Runtime::instance().context(), &p));
            s_ = cuda::own(p, [](owtk_arnoldi_snapshot* q) { owtk_arnoldi_snapshot_destroy(q); });
        }
        owned_ = owned;
        ghost_ = ghost;
        bs_ = bs;
        cache_.clear();
        return s_.get();
    }

private:
    std::shared_ptr<owtk_arnoldi_snapshot> s_;
    std::size_t owned_ = 0, ghost_ = 0, bs_ = 0;
    mutable std::vector<BlockVector<T>> cache_;
};

// ------------------------------------------------------------------ solvers
namespace detail {

template<class Op>
concept DeviceOperator = requires(Op& op) { op.matrix().device(); };

// An application operator or preconditioner (any type with apply(in, out),
// docs/MANUAL.tex:676-712) behind a C callback; errors it throws are kept and
// rethrown by the solver call.
template<std::floating_point T>
struct HostCallbacks {
    std::size_t owned = 0, ghost = 0, bs = 0;
    std::function<void(BlockVector<T>&, BlockVector<T>&)> op, pc;
    const std::function<bool(std::size_t, const BlockVector<T>&)>* test = nullptr;
    std::exception_ptr error;

    BlockVector<T> view(void* p, std::size_t count) const
    {
        return BlockVector<T>::view(owned, ghost, bs, std::span<T>(static_cast<T*>(p), count));
    }
    static int apply_op(void* user, void* in, void* out, size_t count)
    {
        auto* h = static_cast<HostCallbacks*>(user);
        try {
            auto vi = h->view(in, count), vo = h->view(out, count);
            h->op(vi, vo);
            return 0;
        } catch (...) {
            h->error = std::current_exception();
            return 1;
        }
    }
    static int apply_pc(void* user, void* in, void* out, size_t count)
    {
        auto* h = static_cast<HostCallbacks*>(user);
        try {
            auto vi = h->view(in, count), vo = h->view(out, count);
            h->pc(vi, vo);
            return 0;
        } catch (...) {
            h->error = std::current_exception();
            return 1;
        }
    }
    static int convergence(void* user, uint64_t iteration, const void* candidate, size_t count)
    {
        auto* h = static_cast<HostCallbacks*>(user);
        try {
            const auto v = h->view(const_cast<void*>(candidate), count);
            return (*h->test)(static_cast<std::size_t>(iteration), v) ? 1 : 0;
        } catch (...) {
            h->error = std::current_exception();
            return -1;
        }
    }
};

template<std::floating_point T, class Op, class P, class Reduction>
SolverResult<T> device_solve(owtk_solver_kind kind, Op& op, const BlockVector<T>& rhs, BlockVector<T>& x,
                             const SolverOptions<T>& o, P& pc, SolverWorkspace<T>* workspace,
                             ArnoldiSnapshot<T>* snapshot = nullptr)
{
    SolverResult<T> result;
    const auto t0 = std::chrono::steady_clock::now();
    owtk_solver_options co;
    owtk_default_options(&co);
    co.relative_tolerance = static_cast<double>(o.relative_tolerance);
    co.absolute_tolerance = static_cast<double>(o.absolute_tolerance);
    co.breakdown_tolerance = static_cast<double>(o.breakdown_tolerance);
    co.maximum_iterations = o.maximum_iterations;
    co.convergence_check_interval = o.convergence_check_interval;
    co.restart = o.restart;
    co.residual_replacement_interval = o.residual_replacement_interval;
    co.idr_shadow_space = o.idr_shadow_space;
    co.relaxation = static_cast<double>(o.relaxation);
    co.verify_true_residual = o.verify_true_residual ? 1 : 0;
    co.gmres_orthogonalization = static_cast<std::int32_t>(o.gmres_orthogonalization);
    if (!rhs.same_layout(x)) {
        if (snapshot) snapshot->clear();
        return result;
    }
    HostCallbacks<T> cb;
    cb.owned = rhs.owned_nodes();
    cb.ghost = rhs.ghost_nodes();
    cb.bs = rhs.block_size();
    auto* ctx = cuda::Runtime::instance().context();
    owtk_matrix* mh = nullptr;
    std::shared_ptr<owtk_matrix> temp_op;
    if constexpr (DeviceOperator<Op>) {
        const auto& m = op.matrix();
        if (rhs.owned_nodes() != m.owned_nodes() || rhs.ghost_nodes() != m.ghost_nodes()
            || rhs.block_size() != m.block_size())
            throw std::invalid_argument("BlockCsrMatrix vector layout mismatch");
        mh = m.device();
    } else {
        cb.op = [&op](BlockVector<T>& in, BlockVector<T>& out) { op.apply(in, out); };
        owtk_matrix* p = nullptr;
        cuda::check(owtk_callback_operator_create(ctx, cuda::dtype_of<T>(), cb.owned, cb.ghost, cb.bs,
                                                  &HostCallbacks<T>::apply_op, &cb, &p));
        temp_op = cuda::own(p, [](owtk_matrix* q) { owtk_matrix_destroy(q); });
        mh = p;
    }
    owtk_preconditioner* ph = nullptr;
    std::shared_ptr<owtk_preconditioner> temp_pc;
    if constexpr (requires { pc.device(); }) {
        ph = pc.device();
    } else {
        cb.pc = [&pc](BlockVector<T>& in, BlockVector<T>& out) { pc.apply(static_cast<const BlockVector<T>&>(in), out); };
        owtk_preconditioner* p = nullptr;
        cuda::check(owtk_pc_create_callback(ctx, cuda::dtype_of<T>(), cb.owned, cb.ghost, cb.bs,
                                            &HostCallbacks<T>::apply_pc, &cb, &p));
        temp_pc = cuda::own(p, [](owtk_preconditioner* q) { owtk_pc_destroy(q); });
        ph = p;
    }
    owtk_solve_extras ex{};
    ex.reduction = reduction_kind_of<Reduction>();
    if (o.convergence_test) {
        cb.test = &o.convergence_test;
        ex.convergence_test = &HostCallbacks<T>::convergence;
        ex.convergence_user = &cb;
    }
    if (snapshot) ex.arnoldi_snapshot = snapshot->device_for(cb.owned, cb.ghost, cb.bs);
    SolverWorkspace<T> local;
    SolverWorkspace<T>& ws = workspace ? *workspace : local;
    owtk_solver_result r{};
    const owtk_status st = owtk_solve_host_ex(kind, mh, ph, rhs.data(), x.data(), &co, ws.handle(), &ex, &r);
    if (cb.error) std::rethrow_exception(cb.error);
    cuda::check(st);
    result.status = static_cast<SolverStatus>(r.status);
    result.breakdown_reason = static_cast<BreakdownReason>(r.breakdown_reason);
    result.iterations = r.iterations;
    result.operator_applications = r.operator_applications;
    result.preconditioner_applications = r.preconditioner_applications;
    result.global_reductions = r.global_reductions;
    result.reorthogonalizations = r.reorthogonalizations;
    result.arnoldi_norm_verifications = r.arnoldi_norm_verifications;
    result.initial_residual_norm = static_cast<T>(r.initial_residual_norm);
    result.recursive_residual_norm = static_cast<T>(r.recursive_residual_norm);
    result.true_residual_norm = static_cast<T>(r.true_residual_norm);
    result.relative_residual_norm = static_cast<T>(r.relative_residual_norm);
    result.converged_by_application = r.converged_by_application != 0;
    if (o.collect_timings) {
        result.timings = std::make_shared<SolverTimings<T>>();
        result.timings->solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return result;
}

}  // namespace detail

// fgmres / gmres (krylov_solvers.hpp:159-540): fgmres alone records an Arnoldi snapshot.
template<std::floating_point T, class Operator, class Preconditioner = IdentityPreconditioner,
         class Reduction = SerialReduction<T>>
[[nodiscard]] SolverResult<T> fgmres(Operator& op, const BlockVector<T>& rhs, BlockVector<T>& solution,
                                     const SolverOptions<T>& options = {},
                                     Preconditioner&& preconditioner = Preconditioner{}, Reduction = {},
                                     SolverWorkspace<T>* workspace = nullptr,
                                     ArnoldiSnapshot<T>* arnoldi_snapshot = nullptr)
{
    return detail::device_solve<T, Operator, std::remove_reference_t<Preconditioner>, Reduction>(
        OWTK_SOLVER_FGMRES, op, rhs, solution, options, preconditioner, workspace, arnoldi_snapshot);
}

#define OWTK_SOLVER(NAME, KIND)                                                                               \
    template<std::floating_point T, class Operator, class Preconditioner = IdentityPreconditioner,             \
             class Reduction = SerialReduction<T>>                                                             \
    [[nodiscard]] SolverResult<T> NAME(Operator& op, const BlockVector<T>& rhs, BlockVector<T>& solution,      \
                                       const SolverOptions<T>& options = {},                                   \
                                       Preconditioner&& preconditioner = Preconditioner{}, Reduction = {},     \
                                       SolverWorkspace<T>* workspace = nullptr)                                \
    {                                                                                                          \
        return detail::device_solve<T, Operator, std::remove_reference_t<Preconditioner>, Reduction>(         \
            KIND, op, rhs, solution, options, preconditioner, workspace);                                      \
    }

OWTK_SOLVER(gmres, OWTK_SOLVER_FGMRES)
OWTK_SOLVER(bicgstab, OWTK_SOLVER_BICGSTAB)
OWTK_SOLVER(pipelined_bicgstab, OWTK_SOLVER_PIPELINED_BICGSTAB)
OWTK_SOLVER(communication_hiding_bicgstab, OWTK_SOLVER_COMM_HIDING_BICGSTAB)
#undef OWTK_SOLVER

#define OWTK_SOLVER_WITH_WORKSPACE(NAME, KIND)                                                                \
    template<std::floating_point T, class Operator, class Preconditioner = IdentityPreconditioner,             \
             class Reduction = SerialReduction<T>>                                                             \
    [[nodiscard]] SolverResult<T> NAME##_with_workspace(Operator& op, const BlockVector<T>& rhs,               \
                                                        BlockVector<T>& solution, SolverWorkspace<T>& workspace, \
                                                        const SolverOptions<T>& options = {},                  \
                                                        Preconditioner&& preconditioner = Preconditioner{},    \
                                                        Reduction = {})                                        \
    {                                                                                                          \
        return detail::device_solve<T, Operator, std::remove_reference_t<Preconditioner>, Reduction>(         \
            KIND, op, rhs, solution, options, preconditioner, &workspace);                                     \
    }

OWTK_SOLVER_WITH_WORKSPACE(fgmres, OWTK_SOLVER_FGMRES)
OWTK_SOLVER_WITH_WORKSPACE(gmres, OWTK_SOLVER_FGMRES)
OWTK_SOLVER_WITH_WORKSPACE(bicgstab, OWTK_SOLVER_BICGSTAB)
OWTK_SOLVER_WITH_WORKSPACE(pipelined_bicgstab, OWTK_SOLVER_PIPELINED_BICGSTAB)
OWTK_SOLVER_WITH_WORKSPACE(communication_hiding_bicgstab, OWTK_SOLVER_COMM_HIDING_BICGSTAB)
#undef OWTK_SOLVER_WITH_WORKSPACE

// idrs has no workspace parameter (idrs.hpp:128-138).
template<std::floating_point T, class Operator, class Preconditioner = IdentityPreconditioner,
         class Reduction = SerialReduction<T>>
[[nodiscard]] SolverResult<T> idrs(Operator& op, const BlockVector<T>& rhs, BlockVector<T>& solution,
                                   const SolverOptions<T>& options = {},
                                   Preconditioner&& preconditioner = Preconditioner{}, Reduction = {})
{
    return detail::device_solve<T, Operator, std::remove_reference_t<Preconditioner>, Reduction>(
        OWTK_SOLVER_IDRS, op, rhs, solution, options, preconditioner, static_cast<SolverWorkspace<T>*>(nullptr));
}

// The stability variants (krylov_solvers.hpp:766-809, pipelined_bicgstab.hpp:275-313, :620-661):
// the same solvers with the reference's option and reduction choices.
template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> bicgstab_stable(Operator& op, const BlockVector<T>& rhs, BlockVector<T>& solution,
                                              SolverOptions<T> options, Preconditioner&& preconditioner)
{
    options.verify_true_residual = true;
    return bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                    MixedPrecisionSerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner = IdentityPreconditioner,
         class Reduction = SerialReduction<T>>
[[nodiscard]] SolverResult<T> bicgstab_residual_replacement(Operator& op, const BlockVector<T>& rhs,
                                                            BlockVector<T>& solution, SolverOptions<T> options,
                                                            std::size_t replacement_interval,
                                                            Preconditioner&& preconditioner = Preconditioner{},
                                                            Reduction reduction = {})
{
    options.residual_replacement_interval = replacement_interval;
    return bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner), std::move(reduction));
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> bicgstab_mixed_precision(Operator& op, const BlockVector<T>& rhs,
                                                       BlockVector<T>& solution, SolverOptions<T> options,
                                                       Preconditioner&& preconditioner)
{
    return bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                    MixedPrecisionSerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> pipelined_bicgstab_stable(Operator& op, const BlockVector<T>& rhs,
                                                        BlockVector<T>& solution, SolverOptions<T> options,
                                                        Preconditioner&& preconditioner)
{
    return pipelined_bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                              MixedPrecisionSerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> pipelined_bicgstab_residual_replacement(Operator& op, const BlockVector<T>& rhs,
                                                                      BlockVector<T>& solution,
                                                                      SolverOptions<T> options,
                                                                      std::size_t replacement_interval,
                                                                      Preconditioner&& preconditioner)
{
    options.residual_replacement_interval = replacement_interval;
    return pipelined_bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                              SerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> pipelined_bicgstab_mixed_precision(Operator& op, const BlockVector<T>& rhs,
                                                                 BlockVector<T>& solution, SolverOptions<T> options,
                                                                 Preconditioner&& preconditioner)
{
    return pipelined_bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                              MixedPrecisionSerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> communication_hiding_bicgstab_stable(Operator& op, const BlockVector<T>& rhs,
                                                                   BlockVector<T>& solution, SolverOptions<T> options,
                                                                   Preconditioner&& preconditioner)
{
    return communication_hiding_bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                                         MixedPrecisionSerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> communication_hiding_bicgstab_residual_replacement(
    Operator& op, const BlockVector<T>& rhs, BlockVector<T>& solution, SolverOptions<T> options,
    std::size_t replacement_interval, Preconditioner&& preconditioner)
{
    options.residual_replacement_interval = replacement_interval;
    return communication_hiding_bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                                         SerialReduction<T>{});
}

template<std::floating_point T, class Operator, class Preconditioner>
[[nodiscard]] SolverResult<T> communication_hiding_bicgstab_mixed_precision(Operator& op, const BlockVector<T>& rhs,
                                                                            BlockVector<T>& solution,
                                                                            SolverOptions<T> options,
                                                                            Preconditioner&& preconditioner)
{
    return communication_hiding_bicgstab(op, rhs, solution, options, std::forward<Preconditioner>(preconditioner),
                                         MixedPrecisionSerialReduction<T>{});
}

// ------------------------------------------------------------------ SpecWave compatibility
// Legacy SpecWave solver IDs (specwave_compat.hpp:24-48), exact numeric labels.
enum class SpecWaveSolver : int {
    jacobi = 0, gauss_seidel = 1, chebyshev_srj = 2, pipelined_stable = 3, pipelined_residual_replacement = 4,
    bicgstab_ssor = 5, petsc = 6, gmres_ssor = 7, bicgstab_pure_ssor = 8, bicgstab_ilu0 = 9,
    pipelined_mixed_precision = 10, bicgstab_full_system = 11, pipelined_full_system = 12,
    bicgstab_full_system_ilu0 = 13, idrs = 14, communication_hiding_bicgstab = 15, asynchronous_gauss_seidel = 16,
    multigrid_v_jacobi = 17, multigrid_v_red_black = 18, multigrid_w = 19, full_multigrid = 20,
    pipelined_bicgstab_ilu0 = 21, async_pipe_stable = 22,
};

// solve_specwave_native (specwave_compat.hpp:99-249) with the device solvers:
// the same ID -> solver / preconditioner / reduction selection (ID 10 the
// mixed-precision reduction, ID 22 the compensated one).  The stationary and
// multigrid IDs are not on the device path and throw std::invalid_argument;
// PETSc (6) returns a default SolverResult as the reference does.
template<std::floating_point T, std::integral Index, class Operator, class Halo,
         class Reduction = SerialReduction<T>>
[[nodiscard]] SolverResult<T> solve_specwave_native(SpecWaveSolver solver, const BlockCsrMatrix<T, Index>& matrix,
                                                    Operator& linear_operator, Halo&, const BlockVector<T>& rhs,
                                                    BlockVector<T>& solution, SolverOptions<T> options = {},
                                                    Reduction reduction = {})
{
    using S = SpecWaveSolver;
    switch (solver) {
    case S::pipelined_stable:
        return communication_hiding_bicgstab(linear_operator, rhs, solution, options,
                                             LocalSsorPreconditioner<T, Index>(matrix, options.relaxation), reduction);
    case S::pipelined_mixed_precision:
        return communication_hiding_bicgstab(linear_operator, rhs, solution, options,
                                             LocalSsorPreconditioner<T, Index>(matrix, options.relaxation),
                                             MixedPrecisionSerialReduction<T>{});
    case S::async_pipe_stable:
        return communication_hiding_bicgstab(linear_operator, rhs, solution, options,
                                             LocalSsorPreconditioner<T, Index>(matrix, options.relaxation),
                                             CompensatedSerialReduction<T>{});
    case S::pipelined_residual_replacement:
        if (options.residual_replacement_interval == 0) options.residual_replacement_interval = 50;
        return communication_hiding_bicgstab(linear_operator, rhs, solution, options,
                                             LocalSsorPreconditioner<T, Index>(matrix, options.relaxation), reduction);
    case S::bicgstab_ssor:
    case S::bicgstab_pure_ssor:
    case S::bicgstab_full_system:
        return bicgstab(linear_operator, rhs, solution, options,
                        LocalSsorPreconditioner<T, Index>(matrix, options.relaxation), reduction);
    case S::gmres_ssor:
        return gmres(linear_operator, rhs, solution, options,
                     LocalSsorPreconditioner<T, Index>(matrix, options.relaxation), reduction);
    case S::bicgstab_ilu0:
    case S::bicgstab_full_system_ilu0:
        return bicgstab(linear_operator, rhs, solution, options, Ilu0Preconditioner<T, Index>(matrix), reduction);
    case S::pipelined_full_system:
    case S::communication_hiding_bicgstab:
        return pipelined_bicgstab(linear_operator, rhs, solution, options,
                                  LocalSsorPreconditioner<T, Index>(matrix, options.relaxation), reduction);
    case S::idrs:
        return idrs(linear_operator, rhs, solution, options,
                    LocalSsorPreconditioner<T, Index>(matrix, options.relaxation), reduction);
    case S::pipelined_bicgstab_ilu0:
        return pipelined_bicgstab(linear_operator, rhs, solution, options, Ilu0Preconditioner<T, Index>(matrix),
                                  reduction);
    case S::petsc:
        return {};
    default:
        throw std::invalid_argument("SpecWave solver is not on the device path (stationary or multigrid)");
    }
}

// ------------------------------------------------------------------ orderings
template<std::floating_point T, std::integral Index>
[[nodiscard]] std::vector<std::size_t> reverse_cuthill_mckee_order(const BlockCsrMatrix<T, Index>& matrix)
{
    const auto rp = detail::widen<Index>(matrix.row_offsets());
    auto ci = detail::widen<Index>(matrix.column_indices());
    if (ci.empty()) ci.push_back(0);
    std::vector<std::uint64_t> out(matrix.owned_nodes());
    cuda::check(owtk_rcm_order(matrix.owned_nodes(), matrix.ghost_nodes(), rp.data(), ci.data(), out.data()));
    return {out.begin(), out.end()};
}

[[nodiscard]] inline std::vector<std::size_t> hilbert_order(std::span<const std::pair<double, double>> coordinates)
{
    std::vector<double> xy;
    xy.reserve(2 * coordinates.size());
    for (const auto& [x, y] : coordinates) { xy.push_back(x); xy.push_back(y); }
    std::vector<std::uint64_t> out(coordinates.size());
    cuda::check(owtk_hilbert_order(coordinates.size(), xy.data(), out.data()));
    return {out.begin(), out.end()};
}

[[nodiscard]] inline std::vector<std::size_t> inverse_permutation(std::span<const std::size_t> new_to_old)
{
    std::vector<std::uint64_t> in(new_to_old.begin(), new_to_old.end()), out(new_to_old.size());
    cuda::check(owtk_inverse_permutation(in.size(), in.data(), out.data()));
    return {out.begin(), out.end()};
}

// ------------------------------------------------------------------ vector ops (core.hpp:562-601)
// Owned entries only; the arithmetic runs on the device with the reference's
// rounding (no contraction of a*b+c), ghosts are left untouched.
template<std::floating_point T>
inline void copy_owned(const BlockVector<T>& s, BlockVector<T>& d)
{
    if (!s.same_layout(d)) throw std::invalid_argument("BlockVector layout mismatch");
    std::copy(s.owned().begin(), s.owned().end(), d.owned().begin());
}

namespace detail {
// Upload x and y (owned parts), run `op` on the device pair, download y.
template<std::floating_point T, class F>
void device_pair(const BlockVector<T>& x, BlockVector<T>& y, F&& op)
{
    auto [dx, dy] = cuda::Runtime::instance().scratch(cuda::dtype_of<T>(), y.owned_nodes(), y.ghost_nodes(),
                                                      y.block_size());
    cuda::check(owtk_vector_upload(dx, x.data(), x.owned_size()));
    cuda::check(owtk_vector_upload(dy, y.data(), y.owned_size()));
    op(dx, dy);
    cuda::check(owtk_context_synchronize(cuda::Runtime::instance().context()));
    cuda::check(owtk_vector_download(dy, y.data(), y.owned_size()));
}
}  // namespace detail

template<std::floating_point T>
inline void axpy(T alpha, const BlockVector<T>& x, BlockVector<T>& y)
{
    if (!x.same_layout(y)) throw std::invalid_argument("BlockVector layout mismatch");
    detail::device_pair(x, y, [&](owtk_vector* dx, owtk_vector* dy) {
        cuda::check(owtk_axpy(static_cast<double>(alpha), dx, dy));
    });
}

template<std::floating_point T>
inline void scale(T alpha, BlockVector<T>& x)
{
    detail::device_pair(x, x, [&](owtk_vector*, owtk_vector* dy) {
        cuda::check(owtk_scale(static_cast<double>(alpha), dy));
    });
}

template<std::floating_point T>
inline void assign_linear_combination(BlockVector<T>& out, T alpha, const BlockVector<T>& x, T beta,
                                      const BlockVector<T>& y)
{
    if (!out.same_layout(x) || !out.same_layout(y)) throw std::invalid_argument("BlockVector layout mismatch");
    auto [dx, dy] = cuda::Runtime::instance().scratch(cuda::dtype_of<T>(), x.owned_nodes(), x.ghost_nodes(),
                                                      x.block_size());
    cuda::check(owtk_vector_upload(dx, x.data(), x.owned_size()));
    cuda::check(owtk_vector_upload(dy, y.data(), y.owned_size()));
    // The result lands in dx: out = alpha x + beta y, elementwise from the
    // inputs loaded before the store.
    cuda::check(owtk_assign_linear_combination(dx, static_cast<double>(alpha), dx, static_cast<double>(beta), dy));
    cuda::check(owtk_context_synchronize(cuda::Runtime::instance().context()));
    cuda::check(owtk_vector_download(dx, out.data(), out.owned_size()));
}

}  // namespace owt::krylov
