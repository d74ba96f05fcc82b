// Complex GEMM for callers that cannot allocate device memory.
//
// Some callers of this library may not allocate device memory at the point
// where they need a product: a host application whose own allocator has
// reserved the GPU's memory up front (a cudaMalloc from a library inside it
// can fail, or fragment the reserved pool), or a latency-critical loop that
// must not enter the driver's allocation path. tns_zgemm_device_noalloc gives
// them the complex 4M product of tns_zgemm_device without any allocation: its
// working storage -- zero-padded copies of A and B, the product tile target,
// and the 4M partial products P + iQ -- lives in one file-scope device array,
// g_noalloc_scratch, of kNoAllocMaxElements complex elements (64 MiB). The
// array is part of the library's device image, so every GPU that loads the
// library holds it until the process exits.
//
// Host code cannot use the array's name as a device address (on the host it
// names a stand-in). The first call on a device, with that device current,
// looks the address up with cudaGetSymbolAddress once and keeps it; later calls
// on that device reuse it. Every call shares the array and the array keeps the
// previous call's contents, so each call clears the padding it relies on, and
// calls that overlap on the GPU (on different streams or threads) race on it.

#include "tns_internal.h"

#include <mutex>
#include <string>

namespace {

constexpr size_t kNoAllocMaxElements = size_t(1) << 22;  // complex elements, 64 MiB

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocMaxElements];
static __device__ int g_noalloc_error;  // the bounded waits' error flag for these calls

struct DeviceSlot {
    bool ready = false;
    double2* scratch = nullptr;
    int* error = nullptr;
};

std::mutex g_slot_mutex;
DeviceSlot g_slots[64];

// Once per device, with the device current: the arrays' device addresses.
DeviceSlot& device_slot(int device) {
    if (device < 0 || device >= 64) tns::fail(TNS_E_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lock(g_slot_mutex);
    DeviceSlot& s = g_slots[device];
    if (!s.ready) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) tns::fail_cuda(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        s.scratch = static_cast<double2*>(p);
        e = cudaGetSymbolAddress(&p, g_noalloc_error);
        if (e != cudaSuccess) tns::fail_cuda(e, "cudaGetSymbolAddress(g_noalloc_error)", __FILE__, __LINE__);
        s.error = static_cast<int*>(p);
        s.ready = true;
    }
    return s;
}

void require(bool cond, int code, const std::string& msg) {
    if (!cond) tns::fail(code, msg);
}

}  // namespace

extern "C" int tns_zgemm_device_noalloc(void* stream, int m, int n, int k, const double* alpha, const double* a,
                                        int lda, const double* b, int ldb, const double* beta, double* c, int ldc) {
    try {
        require(alpha != nullptr && beta != nullptr, TNS_E_NULL, "alpha or beta is null");
        require(m >= 0 && n >= 0 && k >= 0, TNS_E_ARGUMENT, "negative dimension");
        require(lda >= std::max(1, m) && ldb >= std::max(1, k) && ldc >= std::max(1, m), TNS_E_ARGUMENT,
                "a leading dimension is smaller than its operand's rows");
        require((a || (long long)m * k == 0) && (b || (long long)k * n == 0) && (c || (long long)m * n == 0),
                TNS_E_NULL, "an operand is null");
        if (m == 0 || n == 0) return TNS_OK;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (k == 0) {
            // No product: C := beta*C, as tns_zgemm_device does; alpha is not
            // read, so a non-finite alpha leaves C finite here too.
            tns::scale_detached(s, c, m, n, ldc, true, beta[0], beta[1]);
            TNS_CUDA(cudaStreamSynchronize(s));
            return TNS_OK;
        }
        // Padded extents: the kernel's tiles want M even and K a multiple of 16.
        const size_t mp = (size_t)tns::round_up(m, 2), np = (size_t)tns::round_up(n, 2);
        const size_t kp = (size_t)tns::round_up(k, 16);
        const bool plain = alpha[0] == 1.0 && alpha[1] == 0.0 && beta[0] == 0.0 && beta[1] == 0.0;
        const size_t need = mp * kp + kp * np + mp * np + (plain ? 0 : mp * np);
        if (need > kNoAllocMaxElements)
            tns::fail(TNS_E_OUT_OF_RANGE,
                      "tns_zgemm_device_noalloc: a " + std::to_string(m) + "x" + std::to_string(k) + " by " +
                          std::to_string(k) + "x" + std::to_string(n) + " product needs " + std::to_string(need) +
                          " complex elements of working storage, more than its fixed " +
                          std::to_string(kNoAllocMaxElements) + "; use tns_zgemm_device");
        int device = 0;
        TNS_CUDA(cudaGetDevice(&device));
        DeviceSlot& slot = device_slot(device);

        double2* ap = slot.scratch;
        double2* bp = ap + mp * kp;
        double2* cp = bp + kp * np;
        double2* wp = plain ? nullptr : cp + mp * np;
        // The array keeps the previous call's contents: clear the operands'
        // padding (and everything else in them) before copying in.
        TNS_CUDA(cudaMemsetAsync(ap, 0, (mp * kp + kp * np) * sizeof(double2), s));
        TNS_CUDA(cudaMemcpy2DAsync(ap, mp * sizeof(double2), a, (size_t)lda * sizeof(double2), (size_t)m * sizeof(double2),
                                   k, cudaMemcpyDeviceToDevice, s));
        TNS_CUDA(cudaMemcpy2DAsync(bp, kp * sizeof(double2), b, (size_t)ldb * sizeof(double2), (size_t)k * sizeof(double2),
                                   n, cudaMemcpyDeviceToDevice, s));
        if (!(beta[0] == 0.0 && beta[1] == 0.0))
            TNS_CUDA(cudaMemcpy2DAsync(cp, mp * sizeof(double2), c, (size_t)ldc * sizeof(double2), (size_t)m * sizeof(double2),
                                       n, cudaMemcpyDeviceToDevice, s));
        tns::GemmProblem p{};
        p.A = ap;
        p.B = bp;
        p.C = cp;
        p.lda = (int)mp;
        p.ldb = (int)kp;
        p.ldc = (int)mp;
        p.M = (int)mp;
        p.N = (int)np;
        p.K = (int)kp;
        p.alpha_re = alpha[0];
        p.alpha_im = alpha[1];
        p.beta_re = beta[0];
        p.beta_im = beta[1];
        p.kc = 0;  // the reference's KC for the true size, as tns_zgemm_device
        p.work = (long long)m * n * k;
        p.W = wp;
        p.ldw = (int)mp;
        tns::gemm_detached_complex(s, device, slot.error, p);
        // The product stays in the array until the kernel's wait flag has been
        // read: a wait that gave up leaves the caller's C untouched.
        int flag = 0;
        TNS_CUDA(cudaMemcpyAsync(&flag, slot.error, sizeof(int), cudaMemcpyDeviceToHost, s));
        TNS_CUDA(cudaStreamSynchronize(s));
        if (flag != 0) {
            TNS_CUDA(cudaMemsetAsync(slot.error, 0, sizeof(int), s));
            TNS_CUDA(cudaStreamSynchronize(s));
            tns::fail(TNS_E_TIMEOUT, "a device-side wait gave up (code " + std::to_string(flag) + ")");
        }
        TNS_CUDA(cudaMemcpy2DAsync(c, (size_t)ldc * sizeof(double2), cp, mp * sizeof(double2), (size_t)m * sizeof(double2), n,
                                   cudaMemcpyDeviceToDevice, s));
        TNS_CUDA(cudaStreamSynchronize(s));
        return TNS_OK;
    } catch (const tns::Error& e) {
        tns::set_detached_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        tns::set_detached_error(e.what());
        return TNS_E_DEVICE;
    }
}
