// api.cu — context and particle-buffer entry points of the C ABI.
//
// Particle state is one device allocation holding FPG_FIELD_COUNT 4-byte
// arrays (structure of arrays, each 256-byte aligned).  Upload and download
// move 96-byte fpg_particle records (the reference's Particle,
// src/particles/mod.rs:76-168) through a temporary device buffer and
// transpose on the device, so the host never touches per-field copies.
#include <cuda_runtime.h>

#include <cstring>

#include "fpg_internal.h"

namespace fpg {

static thread_local int32_t g_last_cuda_error = 0;

fpg_status cuda_status(cudaError_t e) {
    g_last_cuda_error = (int32_t)e;
    if (e == cudaErrorMemoryAllocation) return FPG_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoDevice || e == cudaErrorInvalidDevice) return FPG_ERR_NO_DEVICE;
    return FPG_ERR_CUDA;
}

static inline size_t field_stride(size_t capacity) { return ((capacity * 4 + 255) / 256) * 256; }

static void assign_fields(void* block, size_t capacity, void** field) {
    char* b = static_cast<char*>(block);
    const size_t s = field_stride(capacity);
    for (int f = 0; f < FPG_FIELD_COUNT; ++f) field[f] = b + (size_t)f * s;
}

// Record word k (0..23) -> field id, for the 96-byte layout.  Word 23 is pad.
__constant__ int8_t c_word_field[24] = {
    FPG_FIELD_POS_X, FPG_FIELD_POS_Y, FPG_FIELD_POS_Z, FPG_FIELD_CELL_X, FPG_FIELD_CELL_Y, FPG_FIELD_FLAGS,
    FPG_FIELD_MASS0, FPG_FIELD_MASS1, FPG_FIELD_MASS2, FPG_FIELD_MASS3, FPG_FIELD_VEL_U, FPG_FIELD_VEL_V,
    FPG_FIELD_VEL_W, FPG_FIELD_TURB_U, FPG_FIELD_TURB_V, FPG_FIELD_TURB_W, FPG_FIELD_TIME, FPG_FIELD_TIMESTEP,
    FPG_FIELD_TIME_MEM, FPG_FIELD_TIME_SPLIT, FPG_FIELD_RELEASE_POINT, FPG_FIELD_CLASS, FPG_FIELD_CBT, -1};

struct FieldPtrs { uint32_t* f[FPG_FIELD_COUNT]; };

// records (count x 24 words) -> fields at slot (slots ? slots[i] : first + i)
__global__ void __launch_bounds__(256) unpack_kernel(const uint32_t* __restrict__ rec, size_t count, size_t first,
                                                     const uint32_t* __restrict__ slots, FieldPtrs F) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = count * 24;
    if (t >= total) return;
    const size_t i = t / 24;
    const int w = (int)(t - i * 24);
    const int f = c_word_field[w];
    if (f < 0) return;
    const size_t slot = slots ? (size_t)slots[i] : first + i;
    F.f[f][slot] = rec[t];
}

__global__ void __launch_bounds__(256) pack_kernel(uint32_t* __restrict__ rec, size_t count, size_t first,
                                                   FieldPtrs F) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = count * 24;
    if (t >= total) return;
    const size_t i = t / 24;
    const int w = (int)(t - i * 24);
    const int f = c_word_field[w];
    rec[t] = f < 0 ? 0u : F.f[f][first + i];
}

static FieldPtrs field_ptrs(fpg_particles* p) {
    FieldPtrs F;
    for (int f = 0; f < FPG_FIELD_COUNT; ++f) F.f[f] = static_cast<uint32_t*>(p->field[f]);
    return F;
}

static void note_species(fpg_particles* p, const fpg_particle* rec, size_t n) {
    for (size_t i = 0; i < n; ++i)
        for (int k = FPG_MAX_SPECIES - 1; k >= p->n_species; --k)
            if (rec[i].mass[k] != 0.0f) { p->n_species = k + 1; break; }
}

}  // namespace fpg

using namespace fpg;

extern "C" const char* fpg_status_string(fpg_status s) {
    switch (s) {
        case FPG_OK: return "ok";
        case FPG_ERR_INVALID_ARGUMENT: return "invalid argument";
        case FPG_ERR_INVALID_TIME_STEP: return "invalid time step";
        case FPG_ERR_ZERO_SHAPE: return "shape must be non-zero";
        case FPG_ERR_VALUE_TOO_LARGE: return "value does not fit in u32";
        case FPG_ERR_LENGTH_MISMATCH: return "length mismatch";
        case FPG_ERR_INVALID_SPECIES: return "species index out of range";
        case FPG_ERR_INVALID_MASS_SCALE: return "invalid mass scale";
        case FPG_ERR_INVALID_REFERENCE_HEIGHT: return "invalid reference height";
        case FPG_ERR_STORE_FULL: return "particle store full";
        case FPG_ERR_SHAPE_MISMATCH: return "shape mismatch";
        case FPG_ERR_NOT_READY: return "input not uploaded";
        case FPG_ERR_INVALID_BRACKET: return "invalid time bracket";
        case FPG_ERR_OUTSIDE_BRACKET: return "target outside time bracket";
        case FPG_ERR_SIMULATION_COMPLETE: return "simulation complete";
        case FPG_ERR_INVALID_BOUNDS: return "invalid release bounds";
        case FPG_ERR_OUT_OF_GRID: return "release outside grid domain";
        case FPG_ERR_TOO_MANY_LEVELS: return "too many vertical levels";
        case FPG_ERR_INVALID_TIME_RANGE: return "start time after end time";
        case FPG_ERR_INVALID_BACKWARD_TIME_RANGE: return "backward run: start time before end time";
        case FPG_ERR_MISSING_RECEPTORS: return "backward run needs at least one receptor";
        case FPG_ERR_INVALID_RECEPTOR: return "invalid receptor";
        case FPG_ERR_INVALID_SOURCE_BOUNDS: return "invalid source region bounds";
        case FPG_ERR_NON_STOCHASTIC_COLUMN: return "convection matrix column is not stochastic";
        case FPG_ERR_TOO_FEW_LEVELS: return "need at least 2 level interfaces";
        case FPG_ERR_NON_MONOTONIC_INTERFACES: return "level interfaces must be finite and strictly increasing";
        case FPG_ERR_INVALID_BOUNDARY_LAYER_HEIGHT: return "invalid boundary-layer height";
        case FPG_ERR_CUDA: return "CUDA error";
        case FPG_ERR_OUT_OF_MEMORY: return "out of device memory";
        case FPG_ERR_NO_DEVICE: return "no CUDA device";
        default: return "unknown status";
    }
}

extern "C" int32_t fpg_last_cuda_error(void) { return g_last_cuda_error; }
extern "C" int32_t fpg_abi_version(void) { return FPG_ABI_VERSION; }

extern "C" fpg_status fpg_ctx_create(int32_t device, fpg_ctx** out) {
    if (!out) return FPG_ERR_INVALID_ARGUMENT;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return e != cudaSuccess ? cuda_status(e) : FPG_ERR_NO_DEVICE;
    if (device < 0 || device >= n) return FPG_ERR_NO_DEVICE;
    FPG_CUDA(cudaSetDevice(device));
    fpg_ctx* c = new fpg_ctx();
    c->device = device;
    e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        if (c->stream) cudaStreamDestroy(c->stream);
        delete c;
        return cuda_status(e);
    }
    *out = c;
    return FPG_OK;
}

extern "C" fpg_status fpg_ctx_destroy(fpg_ctx* c) {
    if (!c) return FPG_OK;
    cudaStreamSynchronize(c->stream);
    cudaStreamDestroy(c->stream);
    delete c;
    return FPG_OK;
}

extern "C" void* fpg_ctx_stream(fpg_ctx* c) { return c ? c->stream : nullptr; }

extern "C" fpg_status fpg_ctx_synchronize(fpg_ctx* c, void* stream) {
    if (!c) return FPG_ERR_INVALID_ARGUMENT;
    FPG_CUDA(cudaStreamSynchronize(c->pick(stream)));
    return FPG_OK;
}

extern "C" uint64_t fpg_ctx_kernel_launches(fpg_ctx* c) { return c ? c->launches.load() : 0; }

extern "C" fpg_status fpg_device_alloc(fpg_ctx* c, size_t bytes, void** out) {
    if (!c || !out) return FPG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    FPG_CUDA(cudaMalloc(out, bytes > 0 ? bytes : 4));
    return FPG_OK;
}

extern "C" fpg_status fpg_device_free(fpg_ctx* c, void* ptr) {
    if (!c) return FPG_ERR_INVALID_ARGUMENT;
    if (ptr) FPG_CUDA(cudaFree(ptr));
    return FPG_OK;
}

extern "C" fpg_status fpg_host_alloc(fpg_ctx* c, size_t bytes, void** out) {
    if (!c || !out) return FPG_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    FPG_CUDA(cudaHostAlloc(out, bytes > 0 ? bytes : 4, cudaHostAllocDefault));
    return FPG_OK;
}

extern "C" fpg_status fpg_host_free(fpg_ctx* c, void* ptr) {
    if (!c) return FPG_ERR_INVALID_ARGUMENT;
    if (ptr) FPG_CUDA(cudaFreeHost(ptr));
    return FPG_OK;
}

extern "C" fpg_status fpg_memcpy(fpg_ctx* c, void* dst, const void* src, size_t bytes, int32_t kind, void* stream) {
    if (!c || ((!dst || !src) && bytes) || kind < 0 || kind > 2) return FPG_ERR_INVALID_ARGUMENT;
    if (bytes == 0) return FPG_OK;
    static const cudaMemcpyKind kinds[3] = {cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost,
                                            cudaMemcpyDeviceToDevice};
    cudaStream_t s = c->pick(stream);
    FPG_CUDA(cudaMemcpyAsync(dst, src, bytes, kinds[kind], s));
    if (kind == 1) FPG_CUDA(cudaStreamSynchronize(s));
    return FPG_OK;
}

extern "C" fpg_status fpg_memset(fpg_ctx* c, void* dst, int32_t value, size_t bytes, void* stream) {
    if (!c || (!dst && bytes)) return FPG_ERR_INVALID_ARGUMENT;
    if (bytes) FPG_CUDA(cudaMemsetAsync(dst, value, bytes, c->pick(stream)));
    return FPG_OK;
}

extern "C" fpg_status fpg_particles_create(fpg_ctx* ctx, size_t capacity, fpg_particles** out) {
    if (!ctx || !out) return FPG_ERR_INVALID_ARGUMENT;
    if (capacity > (size_t)UINT32_MAX) return FPG_ERR_VALUE_TOO_LARGE;
    fpg_particles* p = new fpg_particles();
    p->ctx = ctx;
    p->capacity = capacity;
    p->dispatch = capacity;
    const size_t bytes = field_stride(capacity > 0 ? capacity : 1) * FPG_FIELD_COUNT;
    cudaError_t e = cudaMalloc(&p->block, bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(p->block, 0, bytes, ctx->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
    if (e != cudaSuccess) {
        cudaFree(p->block);
        delete p;
        return cuda_status(e);
    }
    assign_fields(p->block, capacity > 0 ? capacity : 1, p->field);
    *out = p;
    return FPG_OK;
}

extern "C" fpg_status fpg_particles_destroy(fpg_particles* p) {
    if (!p) return FPG_OK;
    cudaFree(p->block);
    delete p;
    return FPG_OK;
}

extern "C" size_t fpg_particles_capacity(const fpg_particles* p) { return p ? p->capacity : 0; }
extern "C" size_t fpg_particles_dispatch_count(const fpg_particles* p) { return p ? p->dispatch : 0; }

extern "C" fpg_status fpg_particles_set_dispatch_count(fpg_particles* p, size_t count) {
    if (!p) return FPG_ERR_INVALID_ARGUMENT;
    if (count > p->capacity) return FPG_ERR_LENGTH_MISMATCH;
    p->dispatch = count;
    return FPG_OK;
}

static fpg_status upload_records(fpg_particles* p, size_t first, const uint32_t* slots, size_t count,
                                 const fpg_particle* rec, cudaStream_t s) {
    note_species(p, rec, count);
    void* d_rec = nullptr;
    uint32_t* d_slots = nullptr;
    FPG_CUDA(cudaMallocAsync(&d_rec, count * sizeof(fpg_particle), s));
    cudaError_t e = cudaMemcpyAsync(d_rec, rec, count * sizeof(fpg_particle), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && slots) {
        e = cudaMallocAsync(&d_slots, count * sizeof(uint32_t), s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_slots, slots, count * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
    }
    if (e == cudaSuccess) {
        const size_t total = count * 24;
        unpack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(static_cast<const uint32_t*>(d_rec), count,
                                                                      first, d_slots, field_ptrs(p));
        p->ctx->count();
        e = cudaGetLastError();
    }
    cudaFreeAsync(d_rec, s);
    if (d_slots) cudaFreeAsync(d_slots, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host records may be freed after return
    return e == cudaSuccess ? FPG_OK : cuda_status(e);
}

extern "C" fpg_status fpg_particles_upload(fpg_particles* p, size_t first, size_t count, const fpg_particle* rec,
                                           void* stream) {
    if (!p || (!rec && count)) return FPG_ERR_INVALID_ARGUMENT;
    if (first > p->capacity || count > p->capacity - first) return FPG_ERR_LENGTH_MISMATCH;
    if (count == 0) return FPG_OK;
    return upload_records(p, first, nullptr, count, rec, p->ctx->pick(stream));
}

extern "C" fpg_status fpg_particles_upload_slots(fpg_particles* p, const uint32_t* slots, size_t count,
                                                 const fpg_particle* rec, void* stream) {
    if (!p || ((!rec || !slots) && count)) return FPG_ERR_INVALID_ARGUMENT;
    for (size_t i = 0; i < count; ++i)
        if (slots[i] >= p->capacity) return FPG_ERR_LENGTH_MISMATCH;
    if (count == 0) return FPG_OK;
    return upload_records(p, 0, slots, count, rec, p->ctx->pick(stream));
}

extern "C" fpg_status fpg_particles_download(fpg_particles* p, size_t first, size_t count, fpg_particle* out,
                                             void* stream) {
    if (!p || (!out && count)) return FPG_ERR_INVALID_ARGUMENT;
    if (first > p->capacity || count > p->capacity - first) return FPG_ERR_LENGTH_MISMATCH;
    if (count == 0) return FPG_OK;
    cudaStream_t s = p->ctx->pick(stream);
    void* d_rec = nullptr;
    FPG_CUDA(cudaMallocAsync(&d_rec, count * sizeof(fpg_particle), s));
    const size_t total = count * 24;
    pack_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(static_cast<uint32_t*>(d_rec), count, first,
                                                                field_ptrs(p));
    p->ctx->count();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_rec, count * sizeof(fpg_particle), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(d_rec, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? FPG_OK : cuda_status(e);
}

extern "C" void* fpg_particles_field(fpg_particles* p, int32_t field) {
    if (!p || field < 0 || field >= FPG_FIELD_COUNT) return nullptr;
    return p->field[field];
}

extern "C" fpg_status fpg_particles_copy_field(fpg_particles* p, int32_t field, size_t first, size_t count,
                                               void* host, int32_t to_device, void* stream) {
    if (!p || field < 0 || field >= FPG_FIELD_COUNT || (!host && count)) return FPG_ERR_INVALID_ARGUMENT;
    if (first > p->capacity || count > p->capacity - first) return FPG_ERR_LENGTH_MISMATCH;
    if (count == 0) return FPG_OK;
    cudaStream_t s = p->ctx->pick(stream);
    char* dev = static_cast<char*>(p->field[field]) + first * 4;
    if (to_device) {
        if (field >= FPG_FIELD_MASS1 && field <= FPG_FIELD_MASS3) {
            const int k = field - FPG_FIELD_MASS0;
            const float* h = static_cast<const float*>(host);
            for (size_t i = 0; i < count && p->n_species <= k; ++i)
                if (h[i] != 0.0f) p->n_species = k + 1;
        }
        FPG_CUDA(cudaMemcpyAsync(dev, host, count * 4, cudaMemcpyHostToDevice, s));
    } else {
        FPG_CUDA(cudaMemcpyAsync(host, dev, count * 4, cudaMemcpyDeviceToHost, s));
        FPG_CUDA(cudaStreamSynchronize(s));
    }
    return FPG_OK;
}

// Used by compaction: swap the particle block with another of equal capacity.
namespace fpg {
void particles_swap_block(fpg_particles* p, void** other_block) {
    void* b = p->block;
    p->block = *other_block;
    *other_block = b;
    assign_fields(p->block, p->capacity > 0 ? p->capacity : 1, p->field);
}
size_t particles_block_bytes(size_t capacity) { return field_stride(capacity > 0 ? capacity : 1) * FPG_FIELD_COUNT; }
void particles_assign_fields(void* block, size_t capacity, void** field) {
    assign_fields(block, capacity > 0 ? capacity : 1, field);
}
}  // namespace fpg
