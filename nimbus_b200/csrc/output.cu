// Device-side output of a resident level: cell-centre velocities
// (stagger_interpolation.cpp), history frames copied out of HBM, and the npy
// files the reference's export writes (npy_writer.cpp).
#include "../../include/nimbus_cuda.h"
#include "context.cuh"
#include "output_host.cuh"
#include "output_kernels.cuh"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include <string>
#include <thread>
#include <vector>

using namespace nimbus;
using namespace nimbus_host;

namespace
{

// Field names of the reference's core volume bindings
// (core_field_binding_array, headless_runtime.cpp:588-600).
const char* const kHistoryNames[kHistoryFields] = {"u", "v", "w", "rho", "p", "theta", "qv", "qc", "qr"};

bool overlaps(const void* a, const void* b, size_t bytes)
{
    if (!a || !b || !bytes) return false;
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x < y + bytes && y < x + bytes;
}

// interpolate_w_face_to_center_impl's argument check (stagger_interpolation.cpp:29-43).
const char* check_ground(const double* g, size_t columns)
{
    for (size_t c = 0; c < columns; ++c)
        if (!std::isfinite(g[c])) return "terrain lower-boundary velocity must contain only finite values";
    return nullptr;
}

// Widest run (4, 2 or 1 cells) that divides nz and keeps every vector access aligned.
int run_width(int nz, std::initializer_list<const void*> ptrs)
{
    for (int V : {4, 2})
    {
        if (nz % V) continue;
        bool aligned = true;
        for (const void* p : ptrs)
            if (p && reinterpret_cast<uintptr_t>(p) % (sizeof(float) * V)) aligned = false;
        if (aligned) return V;
    }
    return 1;
}

nimbus_status launch_centre(nimbus_cuda_context* ctx, cudaStream_t st, const Dims& d, const CentreFields& F)
{
    if (!F.uc && !F.vc && !F.wc) return NIMBUS_OK;
    const int V = run_width(d.nz, {F.u, F.v, F.w, F.uc, F.vc, F.wc});
    const int grid = grid_for(ctx, d.cells() / V);
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_OUTPUT);
        if (V == 4)
            cell_centre_kernel<4><<<grid, kThreads, 0, st>>>(d, F);
        else if (V == 2)
            cell_centre_kernel<2><<<grid, kThreads, 0, st>>>(d, F);
        else
            cell_centre_kernel<1><<<grid, kThreads, 0, st>>>(d, F);
        ctx->launches += 1;
    }
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

// The ground profile on the device, staged through the context workspace.
nimbus_status stage_ground(nimbus_cuda_context* ctx, cudaStream_t st, const double* host, size_t columns,
                           double** dev)
{
    NB_TRY(ensure(ctx, kGround, columns, dev));
    NB_CUDA(ctx, cudaMemcpyAsync(*dev, host, columns * sizeof(double), cudaMemcpyHostToDevice, st));
    return NIMBUS_OK;
}

}  // namespace

namespace nimbus_host
{

nimbus_status enqueue_history(nimbus_cuda_context* ctx, cudaStream_t st, const float* const src[kHistoryFields],
                              unsigned fields, const double* ground, int nx, int ny, int nz, float* staging,
                              float* host_image)
{
    const Dims d = make_dims(nx, ny, nz);
    const size_t n = static_cast<size_t>(d.cells());
    // The selected velocity components land back to back in staging, in
    // image order, so that they leave the device in one copy.
    const float* from[kHistoryFields] = {};
    CentreFields F{};
    float** outs[3] = {&F.uc, &F.vc, &F.wc};
    const float** ins[3] = {&F.u, &F.v, &F.w};
    int staged = 0;
    for (int f = 0; f < 3; ++f)
    {
        if (!(fields & (1u << f))) continue;
        *ins[f] = src[f];
        *outs[f] = staging + static_cast<size_t>(staged++) * n;
        from[f] = *outs[f];
    }
    F.ground = ground;
    NB_TRY(launch_centre(ctx, st, d, F));
    for (int f = 3; f < kHistoryFields; ++f)
        if (fields & (1u << f)) from[f] = src[f];
    // One copy for the staged velocities (one allocation), one per scalar
    // field: a copy may not span two allocations, and adjacent caller
    // buffers can belong to different ones.
    size_t slot = 0;
    for (int f = 0; f < kHistoryFields;)
    {
        if (!(fields & (1u << f)))
        {
            ++f;
            continue;
        }
        int last = f;
        while (last + 1 < 3 && (fields & (1u << (last + 1))) && from[last + 1] == from[last] + n) ++last;
        const size_t count = static_cast<size_t>(last - f + 1);
        NB_CUDA(ctx, cudaMemcpyAsync(host_image + slot * n, from[f], count * n * sizeof(float),
                                     cudaMemcpyDeviceToHost, st));
        slot += count;
        f = last + 1;
    }
    return NIMBUS_OK;
}

}  // namespace nimbus_host

extern "C" {

nimbus_status nimbus_cuda_cell_centre_velocity(nimbus_cuda_context* ctx, const nimbus_cell_centre_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (a->nx < 0 || a->ny < 0 || a->nz < 0 || !cells_fit(a->nx, a->ny, a->nz))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid cell-centre grid");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    if ((a->u_centre && !a->u) || (a->v_centre && !a->v) || (a->w_centre && !a->w))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "a selected component has no face field");
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const size_t bytes = n * sizeof(float);
    const void* ins[3] = {a->u, a->v, a->w};
    void* outs[3] = {a->u_centre, a->v_centre, a->w_centre};
    for (int o = 0; o < 3; ++o)
    {
        for (int i = 0; i < 3; ++i)
            if (outs[o] && overlaps(outs[o], ins[i], bytes))
                return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "a centre output overlaps a face input");
        for (int p = 0; p < o; ++p)
            if (overlaps(outs[o], outs[p], bytes))
                return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "centre outputs overlap");
    }
    const size_t columns = static_cast<size_t>(a->nx) * a->ny;
    const bool terrain = a->w_centre && a->ground_w;
    if (terrain)
        if (const char* why = check_ground(a->ground_w, columns)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (n == 0 || (!a->u_centre && !a->v_centre && !a->w_centre)) return NIMBUS_OK;

    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE && a->stream) st = static_cast<cudaStream_t>(a->stream);
    double* ground = nullptr;
    if (terrain) NB_TRY(stage_ground(ctx, st, a->ground_w, columns, &ground));
    const Dims d = make_dims(a->nx, a->ny, a->nz);
    if (a->memory == NIMBUS_MEMORY_DEVICE)
        return launch_centre(ctx, st, d, CentreFields{a->u_centre ? a->u : nullptr, a->v_centre ? a->v : nullptr,
                                                      a->w_centre ? a->w : nullptr, a->u_centre, a->v_centre,
                                                      a->w_centre, ground});
    // Host memory: stage the selected faces, centre, copy back.
    const Slot in_slot[3] = {kU, kV, kW};
    float* dev_in[3] = {};
    float* stage = nullptr;
    NB_TRY(ensure(ctx, kCentre, 3 * n, &stage));
    float* dev_out[3] = {};
    for (int f = 0; f < 3; ++f)
    {
        if (!outs[f]) continue;
        NB_TRY(ensure(ctx, in_slot[f], n, &dev_in[f]));
        NB_TRY(upload(ctx, dev_in[f], ins[f], bytes));
        dev_out[f] = stage + static_cast<size_t>(f) * n;
    }
    NB_TRY(launch_centre(ctx, st, d,
                         CentreFields{dev_in[0], dev_in[1], dev_in[2], dev_out[0], dev_out[1], dev_out[2], ground}));
    for (int f = 0; f < 3; ++f)
        if (outs[f]) NB_TRY(download(ctx, outs[f], dev_out[f], bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_history_snapshot(nimbus_cuda_context* ctx, const nimbus_history_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (a->nx < 0 || a->ny < 0 || a->nz < 0 || !cells_fit(a->nx, a->ny, a->nz))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid history grid");
    if (a->fields & ~static_cast<unsigned>(NIMBUS_HISTORY_CORE))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown history field bit");
    const float* src[kHistoryFields] = {a->u, a->v, a->w, a->rho, a->p, a->theta, a->qv, a->qc, a->qr};
    for (int f = 0; f < kHistoryFields; ++f)
        if ((a->fields & (1u << f)) && !src[f])
            return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, std::string("history field ") + kHistoryNames[f] + " is null");
    if (a->fields && !a->host_image) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "host_image is null");
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const size_t columns = static_cast<size_t>(a->nx) * a->ny;
    const bool terrain = (a->fields & NIMBUS_HISTORY_W) && a->ground_w;
    if (terrain)
        if (const char* why = check_ground(a->ground_w, columns)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (n == 0 || !a->fields) return NIMBUS_OK;

    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = a->stream ? static_cast<cudaStream_t>(a->stream) : ctx->stream;
    double* ground = nullptr;
    if (terrain) NB_TRY(stage_ground(ctx, st, a->ground_w, columns, &ground));
    float* stage = nullptr;
    NB_TRY(ensure(ctx, kCentre, 3 * n, &stage));
    return enqueue_history(ctx, st, src, a->fields, ground, a->nx, a->ny, a->nz, stage, a->host_image);
}

nimbus_status nimbus_npy_write_3d(const float* data, int dim0, int dim1, int dim2, const char* path)
{
    if (!data || !path || dim0 <= 0 || dim1 <= 0 || dim2 <= 0) return NIMBUS_ERR_INVALID_ARGUMENT;
    // NPY 1.0: magic (6) + version (2) + header length (2), then the dict,
    // space padding and a newline ending on a 16-byte boundary.
    const std::string dict = "{'descr': '<f4', 'fortran_order': False, 'shape': (" + std::to_string(dim0) + ", " +
                             std::to_string(dim1) + ", " + std::to_string(dim2) + "), }";
    const size_t pad = (16 - (10 + dict.size() + 1) % 16) % 16;
    const size_t header_len = dict.size() + pad + 1;
    std::string head("\x93NUMPY\x01\x00", 8);
    head.push_back(static_cast<char>(header_len & 0xff));
    head.push_back(static_cast<char>((header_len >> 8) & 0xff));
    head += dict;
    head.append(pad, ' ');
    head.push_back('\n');
    const size_t payload = static_cast<size_t>(dim0) * static_cast<size_t>(dim1) * static_cast<size_t>(dim2);
    FILE* f = std::fopen(path, "wb");
    if (!f) return NIMBUS_ERR_IO;
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    ok = ok && std::fwrite(data, sizeof(float), payload, f) == payload;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? NIMBUS_OK : NIMBUS_ERR_IO;
}

nimbus_status nimbus_history_write(const float* host_image, unsigned fields, int nx, int ny, int nz,
                                   const char* step_dir)
{
    if (!host_image || !step_dir || nx <= 0 || ny <= 0 || nz <= 0 ||
        (fields & ~static_cast<unsigned>(NIMBUS_HISTORY_CORE)))
        return NIMBUS_ERR_INVALID_ARGUMENT;
    const size_t n = static_cast<size_t>(nx) * ny * nz;
    // The files are independent: one writer thread each, so a frame is
    // written at the file system's aggregate rate rather than one stream's.
    std::vector<std::thread> writers;
    nimbus_status status[kHistoryFields] = {};
    size_t slot = 0;
    for (int f = 0; f < kHistoryFields; ++f)
    {
        if (!(fields & (1u << f))) continue;
        const float* data = host_image + slot++ * n;
        std::string path = std::string(step_dir) + "/" + kHistoryNames[f] + ".npy";
        writers.emplace_back([=, &status, path = std::move(path)] {
            status[f] = nimbus_npy_write_3d(data, nx, ny, nz, path.c_str());
        });
    }
    for (auto& t : writers) t.join();
    for (int f = 0; f < kHistoryFields; ++f)
        if (status[f] != NIMBUS_OK) return status[f];
    return NIMBUS_OK;
}

}  // extern "C"
