// Registers the reference's operator namespace, nabladyn_neighbors, with identical schemas
// (src/nabladyn/neighbors/csrc/ops.cpp:11-41), so an unchanged NeighborList drives our
// kernels. Each op checks its tensors as the reference does
// (src/nabladyn/neighbors/csrc/runtime/entry_points.cu:24-103: TORCH_CHECK, so a bad argument
// raises RuntimeError), then calls the C-ABI of libnabladyn_b200.so on the current stream.

#include <ATen/core/Tensor.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include <cstdint>
#include <string>
#include <utility>

#include "nabladyn_b200.h"

namespace {

void check(const at::Tensor& tensor, const at::Tensor& reference, at::ScalarType dtype,
           const char* name)
{
    TORCH_CHECK(tensor.is_cuda() && tensor.device() == reference.device(), name,
                " must be on the positions' CUDA device");
    TORCH_CHECK(tensor.is_contiguous(), name, " must be contiguous");
    TORCH_CHECK(tensor.scalar_type() == dtype, name, " has the wrong dtype");
}

int dtype_code(const at::Tensor& positions)
{
    const auto dtype = positions.scalar_type();
    TORCH_CHECK(dtype == at::kFloat || dtype == at::kDouble, "positions must be float32 or float64");
    return dtype == at::kFloat ? ND_FLOAT32 : ND_FLOAT64;
}

void succeed(int rc)
{
    TORCH_CHECK(rc == ND_OK, "nabladyn_b200: ", nd_last_error());
}

// The 15 buffers in schema order, checked against the positions, as C-ABI pointers.
nd_neighbor_buffers buffers_for(
    const at::Tensor& positions,
    at::Tensor& dims, at::Tensor& widths, at::Tensor& atom_bin, at::Tensor& bin_counts,
    at::Tensor& bin_offsets, at::Tensor& unordered_ids, at::Tensor& sorted_ids,
    at::Tensor& sorted_positions, at::Tensor& scan_temp, at::Tensor& pair_counts,
    at::Tensor& pair_offsets, at::Tensor& pair_total, at::Tensor& status, at::Tensor& pairs,
    at::Tensor& bits)
{
    const auto dtype = positions.scalar_type();
    dtype_code(positions);
    TORCH_CHECK(positions.dim() == 2 && positions.size(1) == 3, "positions must be [N, 3]");
    const std::int64_t n = positions.size(0);
    check(positions, positions, dtype, "positions");
    check(widths, positions, dtype, "widths");
    check(sorted_positions, positions, dtype, "sorted_positions");
    const std::pair<const at::Tensor*, const char*> integers[] = {
        {&dims, "dims"},           {&atom_bin, "atom_bin"},         {&bin_counts, "bin_counts"},
        {&bin_offsets, "bin_offsets"}, {&unordered_ids, "unordered_ids"},
        {&sorted_ids, "sorted_ids"}, {&pair_counts, "pair_counts"},
        {&pair_offsets, "pair_offsets"}, {&pair_total, "pair_total"}, {&status, "status"},
        {&pairs, "pairs"},         {&bits, "bits"},
    };
    for (const auto& [tensor, name] : integers)
    {
        check(*tensor, positions, at::kInt, name);
    }
    check(scan_temp, positions, at::kByte, "scan_temp");
    TORCH_CHECK(dims.numel() == 3 && widths.numel() == 3 && atom_bin.numel() == n &&
                    unordered_ids.numel() == n && sorted_ids.numel() == n &&
                    sorted_positions.sizes() == positions.sizes() && bin_counts.numel() >= 2 &&
                    bin_offsets.numel() == bin_counts.numel() && pair_counts.numel() == n &&
                    pair_offsets.numel() == n && pair_total.numel() == 1 && status.numel() == 2,
                "the list's buffers do not match the positions");
    TORCH_CHECK(pairs.dim() == 2 && pairs.size(0) == 2 && pairs.size(1) >= 1 &&
                    pairs.size(1) <= INT32_MAX,
                "pairs must be [2, C] with int32 C");
    const std::int64_t words = (n + 31) / 32;
    TORCH_CHECK(bits.numel() == 0 || bits.numel() == n * words,
                "bits must be empty or hold N rows of ceil(N / 32) words");
    nd_neighbor_buffers b{};
    b.dims = dims.data_ptr<std::int32_t>();
    b.widths = widths.data_ptr();
    b.atom_bin = atom_bin.data_ptr<std::int32_t>();
    b.bin_counts = bin_counts.data_ptr<std::int32_t>();
    b.bin_offsets = bin_offsets.data_ptr<std::int32_t>();
    b.num_bin_slots = bin_counts.numel();
    b.unordered_ids = unordered_ids.data_ptr<std::int32_t>();
    b.sorted_ids = sorted_ids.data_ptr<std::int32_t>();
    b.sorted_positions = sorted_positions.data_ptr();
    b.scan_temp = scan_temp.data_ptr<std::uint8_t>();
    b.scan_temp_bytes = scan_temp.numel();
    b.pair_counts = pair_counts.data_ptr<std::int32_t>();
    b.pair_offsets = pair_offsets.data_ptr<std::int32_t>();
    b.pair_total = pair_total.data_ptr<std::int32_t>();
    b.status = status.data_ptr<std::int32_t>();
    b.pairs = pairs.data_ptr<std::int32_t>();
    b.capacity = pairs.size(1);
    b.bits = bits.numel() > 0 ? bits.data_ptr<std::int32_t>() : nullptr;
    b.bits_numel = bits.numel();
    return b;
}

std::int64_t scan_temp_bytes(const at::Tensor& reference, std::int64_t items)
{
    (void)reference;
    std::int64_t bytes = 0;
    succeed(nd_neighbors_scan_temp_bytes(items, &bytes));
    return bytes;
}

#define ND_BUFFER_PARAMS                                                                     \
    at::Tensor &dims, at::Tensor &widths, at::Tensor &atom_bin, at::Tensor &bin_counts,       \
        at::Tensor &bin_offsets, at::Tensor &unordered_ids, at::Tensor &sorted_ids,           \
        at::Tensor &sorted_positions, at::Tensor &scan_temp, at::Tensor &pair_counts,         \
        at::Tensor &pair_offsets, at::Tensor &pair_total, at::Tensor &status, at::Tensor &pairs, \
        at::Tensor &bits
#define ND_BUFFER_ARGS                                                                      \
    dims, widths, atom_bin, bin_counts, bin_offsets, unordered_ids, sorted_ids,              \
        sorted_positions, scan_temp, pair_counts, pair_offsets, pair_total, status, pairs, bits

void count_first_frame(const at::Tensor& positions, const at::Tensor& cell, double radius,
                       ND_BUFFER_PARAMS)
{
    const nd_neighbor_buffers b = buffers_for(positions, ND_BUFFER_ARGS);
    check(cell, positions, positions.scalar_type(), "cell");
    const c10::cuda::CUDAGuard guard(positions.device());
    succeed(nd_neighbors_count_first_frame(dtype_code(positions), positions.data_ptr(),
                                           cell.data_ptr(), positions.size(0), radius, &b,
                                           c10::cuda::getCurrentCUDAStream().stream()));
}

void fill_first_frame(const at::Tensor& positions, const at::Tensor& cell, double radius,
                      ND_BUFFER_PARAMS)
{
    const nd_neighbor_buffers b = buffers_for(positions, ND_BUFFER_ARGS);
    check(cell, positions, positions.scalar_type(), "cell");
    const c10::cuda::CUDAGuard guard(positions.device());
    succeed(nd_neighbors_fill_first_frame(dtype_code(positions), positions.data_ptr(),
                                          cell.data_ptr(), positions.size(0), radius, &b,
                                          c10::cuda::getCurrentCUDAStream().stream()));
}

void update(const at::Tensor& positions, const at::Tensor& cell, double cutoff, double radius,
            at::Tensor& reference_positions, at::Tensor& reference_cell, const at::Tensor& limits,
            at::Tensor& reuse, at::Tensor& rebuild, at::Tensor& rebuild_count, ND_BUFFER_PARAMS)
{
    const auto dtype = positions.scalar_type();
    const nd_neighbor_buffers b = buffers_for(positions, ND_BUFFER_ARGS);
    check(cell, positions, dtype, "cell");
    check(reference_positions, positions, dtype, "reference_positions");
    check(reference_cell, positions, dtype, "reference_cell");
    check(limits, positions, at::kInt, "limits");
    check(reuse, positions, dtype, "reuse");
    check(rebuild, positions, at::kInt, "rebuild");
    check(rebuild_count, positions, at::kInt, "rebuild_count");
    TORCH_CHECK(cell.numel() == 3 && reference_cell.numel() == 3 && limits.numel() == 3 &&
                    reference_positions.sizes() == positions.sizes() && reuse.numel() == 4 &&
                    rebuild.numel() == 1 && rebuild_count.numel() == 1,
                "the list's update buffers do not match the positions");
    nd_reuse_buffers r{};
    r.reference_positions = reference_positions.data_ptr();
    r.reference_cell = reference_cell.data_ptr();
    r.limits = limits.data_ptr<std::int32_t>();
    r.reuse = reuse.data_ptr();
    r.rebuild = rebuild.data_ptr<std::int32_t>();
    r.rebuild_count = rebuild_count.data_ptr<std::int32_t>();
    const c10::cuda::CUDAGuard guard(positions.device());
    succeed(nd_neighbors_update(dtype_code(positions), positions.data_ptr(), cell.data_ptr(),
                                positions.size(0), cutoff, radius, &r, &b,
                                c10::cuda::getCurrentCUDAStream().stream()));
}

}  // namespace

TORCH_LIBRARY(nabladyn_neighbors, m)
{
    const std::string buffers =
        "Tensor(a!) dims, Tensor(b!) widths, Tensor(c!) atom_bin, Tensor(d!) bin_counts, "
        "Tensor(e!) bin_offsets, Tensor(f!) unordered_ids, Tensor(g!) sorted_ids, "
        "Tensor(h!) sorted_positions, Tensor(i!) scan_temp, Tensor(j!) pair_counts, "
        "Tensor(k!) pair_offsets, Tensor(l!) pair_total, Tensor(m!) status, Tensor(n!) pairs, "
        "Tensor(t!) bits";
    m.def("scan_temp_bytes(Tensor reference, int items) -> int");
    const std::string first_frame = "(Tensor positions, Tensor cell, float radius, " + buffers + ") -> ()";
    m.def(("count_first_frame" + first_frame).c_str());
    m.def(("fill_first_frame" + first_frame).c_str());
    m.def(("update(Tensor positions, Tensor cell, float cutoff, float radius, "
           "Tensor(o!) reference_positions, Tensor(p!) reference_cell, Tensor limits, "
           "Tensor(q!) reuse, Tensor(r!) rebuild, Tensor(s!) rebuild_count, " +
           buffers + ") -> ()")
              .c_str());
}

TORCH_LIBRARY_IMPL(nabladyn_neighbors, CUDA, m)
{
    m.impl("count_first_frame", &count_first_frame);
    m.impl("fill_first_frame", &fill_first_frame);
    m.impl("update", &update);
}

TORCH_LIBRARY_IMPL(nabladyn_neighbors, CompositeExplicitAutograd, m)
{
    m.impl("scan_temp_bytes", &scan_temp_bytes);
}
