// accelerator.cu -- the Accelerator plugin of the reference (Src/Interface/Infrastructure/Accelerator.hpp:130-161,
// Src/Infrastructure/Accelerator/CUDA/CUDA.cpp:497-927) behind the C ABI: device buffers filled from a host
// callback, zeroed tiled outputs, nested resource lookup tables, and launches of generic kernels over a launch
// buffer in the reference's layout (include/piper2_b200_device.cuh), ordered by futures (CUDA events).
//
// B200 choices: memory is stream-ordered (cudaMallocAsync / cudaFreeAsync on the accelerator's streams, as the
// reference's cuMemAllocAsync), pinned staging blocks are pooled instead of allocated per buffer (pinned
// allocation and release synchronise the device), kernels are native sm_100a code registered as CUfunctions and
// launched through the driver's cuLaunchKernel, whose address comes from cudaGetDriverEntryPoint so the library
// needs no link against libcuda.
#include <cuda.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "pb2_internal.h"

using namespace pb2;

#define PB2_CUDA(call, what)                                  \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, (what));  \
    } while (0)

namespace {

constexpr uint32_t kDefaultStreams = 4;
// Threads per block of a generic launch (the reference uses the device's limit, CUDA.cpp:881-886; 256 lets
// register-heavy kernels launch and keeps several blocks resident per SM).
constexpr uint32_t kLaunchBlock = 256;

enum ResourceKind { kBuffer = 0, kTiled = 1, kTable = 2 };

// Makes the accelerator's device current for the scope and restores the caller's (Context::makeCurrent).
struct DeviceScope {
    int saved = -1;
    explicit DeviceScope(int device) {
        if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
        if (saved != device) cudaSetDevice(device);
    }
    ~DeviceScope() {
        int now = -1;
        if (saved >= 0 && cudaGetDevice(&now) == cudaSuccess && now != saved) cudaSetDevice(saved);
    }
};

using LaunchKernelFn = CUresult (*)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                                    CUstream, void**, void**);

}  // namespace

struct pb2_future {
    std::atomic<int> refs{ 1 };
    cudaEvent_t event = nullptr;  // null: complete
};

struct pb2_resource {
    std::atomic<int> refs{ 1 };
    int kind = kBuffer;
    pb2_accelerator* acc = nullptr;
    void* raw = nullptr;      // allocation (device)
    uint64_t handle = 0;      // aligned device address
    size_t size = 0;
    std::mutex mu;            // guards `future`
    pb2_future* future = nullptr;          // the last write (upload, memset, marked writer)
    std::vector<pb2_resource*> entries;    // tables: held entries
};

struct pb2_kernel {
    std::atomic<int> refs{ 1 };
    std::string entry;
    CUfunction fn = nullptr;
};

struct pb2_accelerator {
    // one reference for the caller (pb2_acc_destroy drops it) and one per live resource, so resources released
    // after pb2_acc_destroy still find their streams
    std::atomic<int> refs{ 1 };
    int device = 0;
    std::vector<cudaStream_t> streams;
    uint32_t next_stream = 0;
    std::mutex mu;  // registry, staging pool, in-flight list, stream choice
    std::map<std::string, CUfunction> kernels;
    LaunchKernelFn launch = nullptr;
    struct Staging {
        void* ptr;
        size_t size;
    };
    std::vector<Staging> pool;
    // Work whose completion releases what it holds: staging memory and references.
    struct InFlight {
        pb2_future* done;
        Staging staging;
        std::vector<pb2_resource*> resources;
        pb2_kernel* kernel;
    };
    std::vector<InFlight> inflight;
};

namespace {

void future_retain(pb2_future* f) {
    if (f) f->refs.fetch_add(1, std::memory_order_relaxed);
}

void future_drop(pb2_future* f) {
    if (f && f->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) {
        if (f->event) cudaEventDestroy(f->event);
        delete f;
    }
}

void resource_retain(pb2_resource* r) { r->refs.fetch_add(1, std::memory_order_relaxed); }

void reap_locked(pb2_accelerator* acc, bool wait);

void acc_drop(pb2_accelerator* acc) {
    if (acc->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    DeviceScope scope(acc->device);
    for (cudaStream_t s : acc->streams) cudaStreamSynchronize(s);
    {
        std::lock_guard<std::mutex> lk(acc->mu);
        reap_locked(acc, true);
        for (auto& st : acc->pool) cudaFreeHost(st.ptr);
        acc->pool.clear();
    }
    for (cudaStream_t s : acc->streams) cudaStreamDestroy(s);
    delete acc;
}

void resource_drop(pb2_resource* r) {
    if (!r || r->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
    if (r->raw) {
        // stream-ordered release after the resource's last write
        cudaStream_t s = r->acc->streams[0];
        if (r->future && r->future->event) cudaStreamWaitEvent(s, r->future->event, 0);
        cudaFreeAsync(r->raw, s);
    }
    future_drop(r->future);
    for (pb2_resource* e : r->entries) resource_drop(e);
    pb2_accelerator* acc = r->acc;
    delete r;
    acc_drop(acc);
}

void kernel_drop(pb2_kernel* k) {
    if (k && k->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) delete k;
}

// A new future completed by the work queued on `stream` so far.
int record_future(cudaStream_t stream, pb2_future** out) {
    auto* f = new pb2_future;
    cudaError_t e = cudaEventCreateWithFlags(&f->event, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(f->event, stream);
    if (e != cudaSuccess) {
        future_drop(f);
        return cuda_fail(e, "record future");
    }
    *out = f;
    return PB2_OK;
}

// Releases what finished work held (caller holds acc->mu).
void reap_locked(pb2_accelerator* acc, bool wait) {
    auto& v = acc->inflight;
    size_t keep = 0;
    for (size_t i = 0; i < v.size(); ++i) {
        auto& w = v[i];
        if (wait) cudaEventSynchronize(w.done->event);
        else if (cudaEventQuery(w.done->event) != cudaSuccess) {
            cudaGetLastError();  // not ready is no error
            v[keep++] = w;
            continue;
        }
        if (w.staging.ptr) acc->pool.push_back(w.staging);
        for (pb2_resource* r : w.resources) resource_drop(r);
        kernel_drop(w.kernel);
        future_drop(w.done);
    }
    v.resize(keep);
}

// A pinned staging block of at least `size` bytes (caller holds acc->mu).
int staging_locked(pb2_accelerator* acc, size_t size, pb2_accelerator::Staging* out) {
    size_t best = acc->pool.size();
    for (size_t i = 0; i < acc->pool.size(); ++i)
        if (acc->pool[i].size >= size && (best == acc->pool.size() || acc->pool[i].size < acc->pool[best].size))
            best = i;
    if (best < acc->pool.size()) {
        *out = acc->pool[best];
        acc->pool.erase(acc->pool.begin() + (long)best);
        return PB2_OK;
    }
    size_t bytes = 4096;
    while (bytes < size) bytes <<= 1;
    void* p = nullptr;
    PB2_CUDA(cudaMallocHost(&p, bytes), "cudaMallocHost staging");
    *out = { p, bytes };
    return PB2_OK;
}

// The first idle stream, else the next in turn (CUDAContext::selectOne, CUDA.cpp:248-262).
cudaStream_t pick_stream_locked(pb2_accelerator* acc) {
    for (cudaStream_t s : acc->streams) {
        if (cudaStreamQuery(s) == cudaSuccess) return s;
        cudaGetLastError();  // not ready is no error
    }
    cudaStream_t s = acc->streams[acc->next_stream % acc->streams.size()];
    ++acc->next_stream;
    return s;
}

bool valid_alignment(size_t a) { return a != 0 && (a & (a - 1)) == 0; }

// A device allocation on the stream it returns in *stream (work that fills it must be queued there).
int make_device_resource(pb2_accelerator* acc, int kind, size_t size, size_t alignment, pb2_resource** out,
                         cudaStream_t* stream) {
    if (!acc || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "resource: null argument");
    if (size == 0) return fail(PB2_ERR_INVALID_ARGUMENT, "resource: size 0");
    if (!valid_alignment(alignment)) return fail(PB2_ERR_INVALID_ARGUMENT, "resource: alignment is not a power of two");
    auto* r = new pb2_resource;
    r->kind = kind;
    r->acc = acc;
    r->size = size;
    cudaStream_t s;
    {
        std::lock_guard<std::mutex> lk(acc->mu);
        s = pick_stream_locked(acc);
    }
    // the allocation is at least 256-byte aligned; pad only for larger alignments (CUDA.cpp:536-543)
    const size_t pad = alignment > 256 ? alignment : 0;
    cudaError_t e = cudaMallocAsync(&r->raw, size + pad, s);
    if (e != cudaSuccess) {
        delete r;
        return cuda_fail(e, "cudaMallocAsync resource");
    }
    r->handle = ((uint64_t)(uintptr_t)r->raw + alignment - 1) & ~(uint64_t)(alignment - 1);
    acc->refs.fetch_add(1, std::memory_order_relaxed);
    *out = r;
    *stream = s;
    return PB2_OK;
}

// Flattens a table (ResourceLookUpTableInstance::collect, CUDA.cpp:677-697): entries in order, a nested
// table's slot holding the index where its entries start, nested tables appended after their parent's entries.
void collect(const pb2_resource* table, std::vector<uint64_t>& handles, std::vector<pb2_resource*>& reached) {
    std::vector<std::pair<size_t, const pb2_resource*>> nested;
    for (pb2_resource* e : table->entries) {
        if (e->kind == kTable) {
            nested.emplace_back(handles.size(), e);
            handles.push_back(0);
        } else {
            handles.push_back(e->handle);
            reached.push_back(e);
        }
    }
    for (auto& [slot, t] : nested) {
        handles[slot] = handles.size();
        collect(t, handles, reached);
    }
}

size_t arg_data_size(const uint32_t* desc, uint32_t count) {
    size_t n = 0;
    for (uint32_t i = 0; i < count; ++i) n = std::max(n, (size_t)desc[2 * i] + desc[2 * i + 1]);
    return n;
}

}  // namespace

extern "C" {

int pb2_acc_pack_launch(const uint64_t* handles, uint32_t handle_count, const void* arg_data, const uint32_t* arg_desc,
                        uint32_t arg_count, void* dst, size_t dst_size, size_t* needed) {
    if (!needed || (handle_count && !handles) || (arg_count && !arg_desc))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_pack_launch: null argument");
    const size_t data = arg_data_size(arg_desc, arg_count);
    if (data && !arg_data) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_pack_launch: argument data is null");
    const size_t table = 8 + 8 * (size_t)handle_count;
    const size_t body = table + 8 * (size_t)arg_count;
    const size_t total = body + data;
    if (body > UINT32_MAX) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_pack_launch: too many handles or arguments");
    *needed = total;
    if (!dst) return PB2_OK;
    if (dst_size < total) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_pack_launch: destination too small");
    auto* p = static_cast<unsigned char*>(dst);
    const uint32_t head[2] = { (uint32_t)table, (uint32_t)body };
    std::memcpy(p, head, 8);
    if (handle_count) std::memcpy(p + 8, handles, 8 * (size_t)handle_count);
    if (arg_count) std::memcpy(p + table, arg_desc, 8 * (size_t)arg_count);
    if (data) std::memcpy(p + body, arg_data, data);
    return PB2_OK;
}

int pb2_acc_create(uint32_t streams, pb2_accelerator** out) {
    if (!out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_create: null out");
    *out = nullptr;
    int dev = 0;
    PB2_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    int count = 0;
    PB2_CUDA(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (count == 0) return fail(PB2_ERR_CUDA, "No CUDA-capable device.");
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    PB2_CUDA(cudaGetDriverEntryPoint("cuLaunchKernel", &fn, cudaEnableDefault, &q), "cuLaunchKernel entry point");
    if (q != cudaDriverEntryPointSuccess || !fn) return fail(PB2_ERR_CUDA, "cuLaunchKernel is not available");
    auto* acc = new pb2_accelerator;
    acc->device = dev;
    acc->launch = reinterpret_cast<LaunchKernelFn>(fn);
    const uint32_t n = streams ? streams : kDefaultStreams;
    for (uint32_t i = 0; i < n; ++i) {
        cudaStream_t s = nullptr;
        const cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            pb2_acc_destroy(acc);
            return cuda_fail(e, "cudaStreamCreate");
        }
        acc->streams.push_back(s);
    }
    *out = acc;
    return PB2_OK;
}

int pb2_acc_destroy(pb2_accelerator* acc) {
    if (!acc) return PB2_OK;
    {
        DeviceScope scope(acc->device);
        for (cudaStream_t s : acc->streams) cudaStreamSynchronize(s);
        std::lock_guard<std::mutex> lk(acc->mu);
        reap_locked(acc, true);
    }
    acc_drop(acc);
    return PB2_OK;
}

const char* pb2_acc_native_platform(const pb2_accelerator*) { return "NVIDIA CUDA"; }

int pb2_acc_get_info(const pb2_accelerator* acc, int* device, uint32_t* streams) {
    if (!acc) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_get_info: null accelerator");
    if (device) *device = acc->device;
    if (streams) *streams = (uint32_t)acc->streams.size();
    return PB2_OK;
}

int pb2_acc_create_buffer(pb2_accelerator* acc, size_t size, size_t alignment, pb2_fill_fn fill, void* user,
                          pb2_resource** out) {
    if (!acc || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_create_buffer: null argument");
    *out = nullptr;
    DeviceScope scope(acc->device);
    pb2_resource* r = nullptr;
    cudaStream_t s = nullptr;
    int rc = make_device_resource(acc, kBuffer, size, alignment, &r, &s);
    if (rc) return rc;
    std::unique_lock<std::mutex> lk(acc->mu);
    reap_locked(acc, false);
    pb2_accelerator::Staging st{};
    if ((rc = staging_locked(acc, size, &st))) {
        lk.unlock();
        resource_drop(r);
        return rc;
    }
    lk.unlock();
    // the host callback fills the staging block (the reference runs it on its scheduler, CUDA.cpp:522-532)
    if (fill) fill(st.ptr, size, user);
    else std::memset(st.ptr, 0, size);
    pb2_future* f = nullptr;
    cudaError_t e = cudaMemcpyAsync(reinterpret_cast<void*>(r->handle), st.ptr, size, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) rc = record_future(s, &f);
    lk.lock();
    if (e != cudaSuccess || rc) {
        cudaStreamSynchronize(s);
        acc->pool.push_back(st);
        lk.unlock();
        resource_drop(r);
        return e != cudaSuccess ? cuda_fail(e, "buffer upload") : rc;
    }
    r->future = f;
    future_retain(f);
    acc->inflight.push_back({ f, st, {}, nullptr });
    *out = r;
    return PB2_OK;
}

int pb2_acc_create_tiled_output(pb2_accelerator* acc, size_t size, size_t alignment, pb2_resource** out) {
    if (!acc || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_create_tiled_output: null argument");
    *out = nullptr;
    DeviceScope scope(acc->device);
    pb2_resource* r = nullptr;
    cudaStream_t s = nullptr;
    int rc = make_device_resource(acc, kTiled, size, alignment, &r, &s);
    if (rc) return rc;
    // allocation and reset on the same stream (CUDA.cpp:591-602); the memset completes the first future
    cudaError_t e = cudaMemsetAsync(reinterpret_cast<void*>(r->handle), 0, size, s);
    if (e == cudaSuccess) rc = record_future(s, &r->future);
    if (e != cudaSuccess || rc) {
        resource_drop(r);
        return e != cudaSuccess ? cuda_fail(e, "tiled output reset") : rc;
    }
    *out = r;
    return PB2_OK;
}

int pb2_acc_create_resource_lut(pb2_accelerator* acc, pb2_resource* const* resources, uint32_t count,
                                pb2_resource** out) {
    if (!acc || !out || (count && !resources))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_create_resource_lut: null argument");
    for (uint32_t i = 0; i < count; ++i) {
        if (!resources[i]) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_create_resource_lut: null entry");
        if (resources[i]->acc != acc)
            return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_create_resource_lut: entry of another accelerator");
    }
    auto* t = new pb2_resource;
    t->kind = kTable;
    t->acc = acc;
    acc->refs.fetch_add(1, std::memory_order_relaxed);
    for (uint32_t i = 0; i < count; ++i) {
        resource_retain(resources[i]);
        t->entries.push_back(resources[i]);
    }
    *out = t;
    return PB2_OK;
}

int pb2_resource_get_handle(const pb2_resource* res, uint64_t* handle) {
    if (!res || !handle) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_resource_get_handle: null argument");
    // a table has no handle of its own (ResourceLookUpTableInstance::getHandle is notSupported, CUDA.cpp:669-672)
    if (res->kind == kTable) return fail(PB2_ERR_NOT_SUPPORTED, "pb2_resource_get_handle: a lookup table has no handle");
    *handle = res->handle;
    return PB2_OK;
}

int pb2_resource_release(pb2_resource* res) {
    if (!res) return PB2_OK;
    DeviceScope scope(res->acc->device);
    resource_drop(res);
    return PB2_OK;
}

int pb2_tiled_output_mark_dirty(pb2_resource* output, pb2_future* writer) {
    if (!output || !writer) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_tiled_output_mark_dirty: null argument");
    if (output->kind != kTiled) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_tiled_output_mark_dirty: not a tiled output");
    future_retain(writer);
    pb2_future* old;
    {
        std::lock_guard<std::mutex> lk(output->mu);
        old = output->future;
        output->future = writer;
    }
    future_drop(old);
    return PB2_OK;
}

int pb2_tiled_output_download(pb2_resource* output, void* dst_host, size_t size) {
    if (!output || (size && !dst_host)) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_tiled_output_download: null argument");
    if (output->kind != kTiled) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_tiled_output_download: not a tiled output");
    if (size > output->size) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_tiled_output_download: size exceeds the output");
    pb2_accelerator* acc = output->acc;
    DeviceScope scope(acc->device);
    pb2_future* f;
    {
        std::lock_guard<std::mutex> lk(output->mu);
        f = output->future;
        future_retain(f);
    }
    cudaStream_t s;
    {
        std::lock_guard<std::mutex> lk(acc->mu);
        s = pick_stream_locked(acc);
    }
    cudaError_t e = cudaSuccess;
    if (f && f->event) e = cudaStreamWaitEvent(s, f->event, 0);
    future_drop(f);
    if (e == cudaSuccess && size)
        e = cudaMemcpyAsync(dst_host, reinterpret_cast<const void*>(output->handle), size, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "tiled output download");
    return PB2_OK;
}

int pb2_acc_register_kernel(pb2_accelerator* acc, const char* entry, void* cu_function) {
    if (!acc || !entry || !*entry || !cu_function)
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_register_kernel: null argument");
    std::lock_guard<std::mutex> lk(acc->mu);
    acc->kernels[entry] = static_cast<CUfunction>(cu_function);
    return PB2_OK;
}

int pb2_acc_compile_kernel(pb2_accelerator* acc, const char* entry, pb2_kernel** out) {
    if (!acc || !entry || !out) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_compile_kernel: null argument");
    *out = nullptr;
    std::lock_guard<std::mutex> lk(acc->mu);
    const auto it = acc->kernels.find(entry);
    if (it == acc->kernels.end())
        return fail(PB2_ERR_NOT_SUPPORTED, std::string("pb2_acc_compile_kernel: no kernel named \"") + entry + "\"");
    auto* k = new pb2_kernel;
    k->entry = entry;
    k->fn = it->second;
    *out = k;
    return PB2_OK;
}

int pb2_kernel_release(pb2_kernel* kernel) {
    kernel_drop(kernel);
    return PB2_OK;
}

int pb2_acc_launch_kernel(pb2_accelerator* acc, const uint32_t dim[3], pb2_kernel* kernel, pb2_resource* root,
                          const void* arg_data, const uint32_t* arg_desc, uint32_t arg_count, pb2_future** out) {
    if (out) *out = nullptr;
    if (!acc || !dim || !kernel) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_launch_kernel: null argument");
    if (root && (root->kind != kTable || root->acc != acc))
        return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_acc_launch_kernel: root is not a lookup table of this accelerator");
    if (!(dim[0] && dim[1] && dim[2])) return fail(PB2_ERR_INVALID_ARGUMENT, "Empty launch");
    if ((uint64_t)dim[0] * dim[1] * dim[2] > (uint64_t)INT_MAX)
        return fail(PB2_ERR_NOT_SUPPORTED, "pb2_acc_launch_kernel: more than INT_MAX tasks in one launch");
    const uint32_t block = std::min(dim[2], kLaunchBlock);
    const uint32_t gz = (dim[2] + block - 1) / block;
    if (dim[1] > 65535u || gz > 65535u)
        return fail(PB2_ERR_NOT_SUPPORTED, "pb2_acc_launch_kernel: dim[1] or dim[2] / 256 exceeds 65535");
    DeviceScope scope(acc->device);
    // flatten the tables and gather the futures to wait for
    std::vector<uint64_t> handles;
    std::vector<pb2_resource*> reached;
    if (root) collect(root, handles, reached);
    size_t bytes = 0;
    int rc = pb2_acc_pack_launch(handles.data(), (uint32_t)handles.size(), arg_data, arg_desc, arg_count, nullptr, 0,
                                 &bytes);
    if (rc) return rc;
    std::unique_lock<std::mutex> lk(acc->mu);
    reap_locked(acc, false);
    pb2_accelerator::Staging st{};
    if ((rc = staging_locked(acc, bytes, &st))) return rc;
    cudaStream_t s = pick_stream_locked(acc);
    lk.unlock();
    pb2_acc_pack_launch(handles.data(), (uint32_t)handles.size(), arg_data, arg_desc, arg_count, st.ptr, st.size, &bytes);
    cudaError_t e = cudaSuccess;
    for (pb2_resource* r : reached) {
        std::lock_guard<std::mutex> g(r->mu);
        if (r->future && r->future->event && e == cudaSuccess) e = cudaStreamWaitEvent(s, r->future->event, 0);
    }
    void* dbuf = nullptr;
    if (e == cudaSuccess) e = cudaMallocAsync(&dbuf, bytes, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dbuf, st.ptr, bytes, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        uint32_t max_z = dim[2];
        void* params[2] = { &max_z, &dbuf };
        const CUresult cr = acc->launch(kernel->fn, dim[0], dim[1], gz, block, 1, 1, 0, reinterpret_cast<CUstream>(s),
                                        params, nullptr);
        if (cr != CUDA_SUCCESS) {
            cudaFreeAsync(dbuf, s);
            cudaStreamSynchronize(s);
            lk.lock();
            acc->pool.push_back(st);
            return fail(PB2_ERR_CUDA, "pb2_acc_launch_kernel: cuLaunchKernel of \"" + kernel->entry + "\" failed (" +
                                          std::to_string((int)cr) + ")");
        }
        e = cudaFreeAsync(dbuf, s);
    }
    pb2_future* f = nullptr;
    if (e == cudaSuccess) rc = record_future(s, &f);
    lk.lock();
    if (e != cudaSuccess || rc) {
        cudaStreamSynchronize(s);
        acc->pool.push_back(st);
        return e != cudaSuccess ? cuda_fail(e, "pb2_acc_launch_kernel") : rc;
    }
    // the launch holds its kernel, table and resources until it completes
    pb2_accelerator::InFlight w{ f, st, {}, kernel };
    kernel->refs.fetch_add(1, std::memory_order_relaxed);
    if (root) {
        resource_retain(root);
        w.resources.push_back(root);
    }
    acc->inflight.push_back(w);
    if (out) {
        future_retain(f);
        *out = f;
    }
    return PB2_OK;
}

int pb2_future_wait(pb2_future* future) {
    if (!future) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_future_wait: null future");
    if (future->event) PB2_CUDA(cudaEventSynchronize(future->event), "pb2_future_wait");
    return PB2_OK;
}

int pb2_future_ready(pb2_future* future, int* ready) {
    if (!future || !ready) return fail(PB2_ERR_INVALID_ARGUMENT, "pb2_future_ready: null argument");
    if (!future->event) {
        *ready = 1;
        return PB2_OK;
    }
    const cudaError_t e = cudaEventQuery(future->event);
    if (e == cudaErrorNotReady) {
        cudaGetLastError();
        *ready = 0;
        return PB2_OK;
    }
    if (e != cudaSuccess) return cuda_fail(e, "pb2_future_ready");
    *ready = 1;
    return PB2_OK;
}

int pb2_future_release(pb2_future* future) {
    future_drop(future);
    return PB2_OK;
}

}  // extern "C"
