// Context (one CUDA stream per workspace), padded device matrices, transfers.

#include "device_util.cuh"
#include "tns_internal.h"

#include <cstring>
#include <sstream>

namespace tns {

void fail(int code, const std::string& msg) { throw Error(code, msg); }

void fail_cuda(cudaError_t e, const char* what, const char* file, int line) {
    std::ostringstream os;
    os << "CUDA error " << cudaGetErrorName(e) << " (" << cudaGetErrorString(e) << ") in " << what << " at " << file << ":"
       << line;
    int code = (e == cudaErrorMemoryAllocation) ? TNS_E_OUT_OF_MEMORY : TNS_E_DEVICE;
    if (e == cudaErrorMemoryAllocation) cudaGetLastError();  // not sticky; clear it
    throw Error(code, os.str());
}

Context::Context(int dev) : device(dev) {
    int count = 0;
    TNS_CUDA(cudaGetDeviceCount(&count));
    if (dev < 0 || dev >= count) fail(TNS_E_ARGUMENT, "no CUDA device " + std::to_string(dev));
    TNS_CUDA(cudaSetDevice(dev));
    TNS_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev));
    TNS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    TNS_CUDA(cudaMalloc(&d_err, sizeof(int)));
    TNS_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    TNS_CUDA(cudaMalloc(&d_tiles, sizeof(unsigned long long)));
    // Keep freed blocks in the stream-ordered pool instead of handing them back
    // to the driver at every synchronisation: the algorithms allocate and free
    // work matrices between host-side decisions.
    cudaMemPool_t pool;
    TNS_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t keep = ~0ull;
    TNS_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
}

cudaEvent_t Context::take_event() {
    if (event_pool.empty()) {
        cudaEvent_t e;
        TNS_CUDA(cudaEventCreate(&e));
        return e;
    }
    cudaEvent_t e = event_pool.back();
    event_pool.pop_back();
    return e;
}

void Context::drain_events() {
    if (gemm_events.empty() && split_events.empty()) return;
    TNS_CUDA(cudaStreamSynchronize(stream));
    auto drain = [&](std::vector<std::pair<cudaEvent_t, cudaEvent_t>>& evs, double& total) {
        for (auto& pr : evs) {
            float ms = 0.f;
            TNS_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
            total += ms;
            event_pool.push_back(pr.first);
            event_pool.push_back(pr.second);
        }
        evs.clear();
    };
    drain(gemm_events, gemm_ms_done);
    drain(split_events, split_ms_done);
}

Context::~Context() {
    workers.clear();
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (auto* evs : {&gemm_events, &split_events})
        for (auto& pr : *evs) {
            cudaEventDestroy(pr.first);
            cudaEventDestroy(pr.second);
        }
    for (auto e : event_pool) cudaEventDestroy(e);
    if (split_scratch) cudaFree(split_scratch);
    if (h_ring) cudaFreeHost(h_ring);
    if (d_ring) cudaFree(d_ring);
    if (d_err) cudaFree(d_err);
    if (d_tiles) cudaFree(d_tiles);
    if (copy_stream) {
        cudaStreamSynchronize(copy_stream);
        cudaStreamDestroy(copy_stream);
    }
    if (stream) cudaStreamDestroy(stream);
}

cudaStream_t Context::copies() {
    if (!copy_stream) TNS_CUDA(cudaStreamCreateWithFlags(&copy_stream, cudaStreamNonBlocking));
    return copy_stream;
}

const void* Context::upload(const void* src, size_t bytes) {
    size_t need = (bytes + 255) & ~size_t(255);
    if (need > ring_cap) {
        // Grow: everything already queued must finish with the old ring.
        TNS_CUDA(cudaStreamSynchronize(stream));
        if (h_ring) TNS_CUDA(cudaFreeHost(h_ring));
        if (d_ring) TNS_CUDA(cudaFree(d_ring));
        h_ring = nullptr;
        d_ring = nullptr;
        ring_cap = std::max(need, size_t(4) << 20);
        TNS_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&h_ring), ring_cap, cudaHostAllocDefault));
        TNS_CUDA(cudaMalloc(reinterpret_cast<void**>(&d_ring), ring_cap));
        ring_pos = 0;
    }
    if (ring_pos + need > ring_cap) {
        // Wrap around: the copies and kernels still reading the ring finish first.
        TNS_CUDA(cudaStreamSynchronize(stream));
        ring_pos = 0;
    }
    std::memcpy(h_ring + ring_pos, src, bytes);
    TNS_CUDA(cudaMemcpyAsync(d_ring + ring_pos, h_ring + ring_pos, bytes, cudaMemcpyHostToDevice, stream));
    const void* out = d_ring + ring_pos;
    ring_pos += need;
    return out;
}

void Context::sync() { TNS_CUDA(cudaStreamSynchronize(stream)); }

void Context::check_limit(long long elements, const char* purpose) const {
    if (elements > max_elements) {
        std::ostringstream os;
        os << "Refused to allocate " << elements << " elements for " << purpose << ": TensileLimits.MaxElements is "
           << max_elements << ".";
        fail(TNS_E_ALLOCATION_LIMIT, os.str());
    }
}

DMat::DMat(Context& c, int r, int k, bool complex_, const char* purpose)
    : ctx(&c), rows(r), cols(k), rows_p(round_up(std::max(r, 1), kPad)), cols_p(round_up(std::max(k, 1), kPad)),
      cplx(complex_) {
    if (r < 0 || k < 0) fail(TNS_E_ARGUMENT, "negative matrix dimension");
    c.check_limit((long long)r * k, purpose);
    c.count_allocation();
    TNS_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), bytes(), c.stream));
    TNS_CUDA(cudaMemsetAsync(p, 0, bytes(), c.stream));
}

DMat& DMat::operator=(DMat&& o) noexcept {
    if (this != &o) {
        if (p && ctx) cudaFreeAsync(p, ctx->stream);
        ctx = o.ctx;
        p = o.p;
        rows = o.rows;
        cols = o.cols;
        rows_p = o.rows_p;
        cols_p = o.cols_p;
        cplx = o.cplx;
        o.p = nullptr;
        o.ctx = nullptr;
    }
    return *this;
}

DMat::~DMat() {
    if (p && ctx) cudaFreeAsync(p, ctx->stream);
}

void DMat::zero() { TNS_CUDA(cudaMemsetAsync(p, 0, bytes(), ctx->stream)); }

void* Context::scratch(size_t bytes) {
    if (bytes > split_scratch_bytes) {
        if (split_scratch) TNS_CUDA(cudaFreeAsync(split_scratch, stream));
        split_scratch = nullptr;
        split_scratch_bytes = 0;
        const size_t grown = std::max(bytes, bytes + bytes / 4);  // headroom for the next, larger batch
        count_allocation();
        TNS_CUDA(cudaMallocAsync(&split_scratch, grown, stream));
        split_scratch_bytes = grown;
    }
    return split_scratch;
}

DBuf::DBuf(Context& c, size_t b) : ctx(&c), bytes(b) {
    c.count_allocation();
    TNS_CUDA(cudaMallocAsync(&p, std::max<size_t>(b, 16), c.stream));
}

void Context::count_allocation() {
    ++allocations;
    if (fail_allocation_at > 0 && allocations >= fail_allocation_at) {
        fail_allocation_at = 0;  // one injected failure, then allocations succeed again
        fail(TNS_E_OUT_OF_MEMORY, "device allocation " + std::to_string(allocations) +
                                      " refused (injected failure, tns_inject_allocation_failure)");
    }
}

namespace {
// A barrier that nothing ever arrives on: the bounded wait must give up after
// limit_ns, record kDevTimeoutSelfTest and return. Nothing else is in flight.
__global__ void wait_selftest_kernel(int* err, unsigned long long limit_ns) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
    }
    __syncthreads();
    mbar_wait_bounded_ns(&bar, 0, err, kDevTimeoutSelfTest, limit_ns);
}
}  // namespace

void selftest_wait(Context& ctx, long long limit_ns) {
    wait_selftest_kernel<<<1, 32, 0, ctx.stream>>>(ctx.d_err, (unsigned long long)limit_ns);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}
DBuf& DBuf::operator=(DBuf&& o) noexcept {
    if (this != &o) {
        if (p && ctx) cudaFreeAsync(p, ctx->stream);
        ctx = o.ctx;
        p = o.p;
        bytes = o.bytes;
        o.p = nullptr;
        o.ctx = nullptr;
    }
    return *this;
}
DBuf::~DBuf() {
    if (p && ctx) cudaFreeAsync(p, ctx->stream);
}

void copy_in(Context& ctx, DMat& dst, const double* src, int ld, bool src_on_device) {
    if (dst.rows == 0 || dst.cols == 0) return;
    size_t esz = dst.esz();
    TNS_CUDA(cudaMemcpy2DAsync(dst.p, (size_t)dst.ld() * esz, src, (size_t)ld * esz, (size_t)dst.rows * esz, dst.cols,
                               src_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx.stream));
}

void copy_out_on(cudaStream_t stream, const DMat& src, double* dst, int ld, bool dst_on_device) {
    if (src.rows == 0 || src.cols == 0) return;
    size_t esz = src.esz();
    TNS_CUDA(cudaMemcpy2DAsync(dst, (size_t)ld * esz, src.p, (size_t)src.ld() * esz, (size_t)src.rows * esz, src.cols,
                               dst_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, stream));
}

void copy_out(Context& ctx, const DMat& src, double* dst, int ld, bool dst_on_device) {
    copy_out_on(ctx.stream, src, dst, ld, dst_on_device);
}

void copy_dmat(Context& ctx, DMat& dst, const DMat& src) {
    if (dst.bytes() != src.bytes()) fail(TNS_E_ARGUMENT, "internal copy between differently shaped matrices");
    TNS_CUDA(cudaMemcpyAsync(dst.p, src.p, src.bytes(), cudaMemcpyDeviceToDevice, ctx.stream));
}

GemmProblem make_gemm(const DMat& a, const DMat& b, DMat& c, double alpha_re, double alpha_im, double beta_re,
                      double beta_im) {
    if (a.cols != b.rows || c.rows != a.rows || c.cols != b.cols || a.cplx != b.cplx || a.cplx != c.cplx)
        fail(TNS_E_ARGUMENT, "internal product of non-conformable matrices");
    GemmProblem p{};
    p.A = a.p;
    p.B = b.p;
    p.C = c.p;
    p.lda = a.ld();
    p.ldb = b.ld();
    p.ldc = c.ld();
    p.M = round_up(a.rows, 2);
    p.N = round_up(b.cols, 2);
    p.K = round_up(a.cols, 16);
    p.alpha_re = alpha_re;
    p.alpha_im = alpha_im;
    p.beta_re = beta_re;
    p.beta_im = beta_im;
    p.kc = 0;  // the reference's KC for this product's true size
    p.work = (long long)a.rows * b.cols * a.cols;
    p.W = nullptr;
    p.ldw = 0;
    return p;
}

namespace {
// dst(j, i) = conj(src(i, j)) over the padded extents, 32 x 32 tiles.
__global__ void conj_transpose_kernel(double* dst, int ldd, const double* src, int lds, int rows, int cols, bool cplx) {
    __shared__ double2 tile[32][33];
    int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx: src rows, by: src cols
    int tx = threadIdx.x, ty = threadIdx.y;
    for (int k = ty; k < 32; k += blockDim.y) {
        int i = bx + tx, j = by + k;
        double2 v = make_double2(0.0, 0.0);
        if (i < rows && j < cols) {
            if (cplx) v = reinterpret_cast<const double2*>(src)[(size_t)j * lds + i];
            else v.x = src[(size_t)j * lds + i];
        }
        tile[k][tx] = v;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += blockDim.y) {
        int i = by + tx, j = bx + k;  // dst row i (= src col), dst col j (= src row)
        if (i < cols && j < rows) {
            double2 v = tile[tx][k];
            if (cplx) reinterpret_cast<double2*>(dst)[(size_t)j * ldd + i] = make_double2(v.x, -v.y);
            else dst[(size_t)j * ldd + i] = v.x;
        }
    }
}
}  // namespace

void conj_transpose(Context& ctx, DMat& dst, const DMat& src) {
    dim3 grid((src.rows_p + 31) / 32, (src.cols_p + 31) / 32);
    conj_transpose_kernel<<<grid, dim3(32, 8), 0, ctx.stream>>>(dst.p, dst.ld(), src.p, src.ld(), src.rows_p, src.cols_p,
                                                               src.cplx);
    TNS_CUDA(cudaGetLastError());
    ctx.kernel_launches++;
}

}  // namespace tns
