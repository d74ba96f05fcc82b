// Launch-parameter plumbing shared by the kernels that run either on one
// matrix or on a whole batch in one launch: a kernel receives a Batch<D>; the
// item index (blockIdx.y, or blockIdx.x for one-CTA-per-item kernels) selects
// a descriptor D, which travels inline for a single item and in device memory
// for a batch.
#pragma once

#include <vector>

#include "tns_internal.h"

namespace tns {

template <class D>
struct Batch {
    D one;
    const D* list;
    int count;
};

template <class D>
__device__ __forceinline__ const D& batch_item(const Batch<D>& b, int i) {
    return b.list ? b.list[i] : b.one;
}

template <class D>
Batch<D> make_batch(Context& ctx, const std::vector<D>& v) {
    Batch<D> b{};
    b.count = (int)v.size();
    if (v.size() == 1) {
        b.one = v[0];
        b.list = nullptr;
    } else if (!v.empty()) {
        b.list = static_cast<const D*>(ctx.upload(v.data(), sizeof(D) * v.size()));
    }
    return b;
}

template <class D>
Batch<D> single(const D& d) {
    Batch<D> b{};
    b.one = d;
    b.list = nullptr;
    b.count = 1;
    return b;
}

}  // namespace tns
