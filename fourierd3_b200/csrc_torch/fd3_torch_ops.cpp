// Thin PyTorch operator layer over the C ABI of libfd3 (include/fd3.h): registers
// torch.ops.fd3.energy_forces_stress (the fused E+F+stress call behind the functional
// forward / FourierD3ASECalculator.calculate, src/fourierd3/calculator.py:125-192) and
// torch.ops.fd3.energy_edges (the module path behind FourierD3.forward with caller edges,
// src/fourierd3/core.py:480-583), with CUDA kernels that call libfd3 on the current stream and
// Meta kernels that give output shapes (so the ops trace under torch.compile / export). The
// plan (tables, cuFFT plans) is created through the same C ABI and passed as an integer handle.
// Everything numerical happens in libfd3; this file only checks tensors and forwards pointers.
#include <ATen/ATen.h>
#include <c10/cuda/CUDAGuard.h>
#include <c10/cuda/CUDAStream.h>
#include <torch/library.h>

#include "fd3.h"

namespace {

void check_cuda(const at::Tensor& t, at::ScalarType dt, const char* name) {
  TORCH_CHECK(t.is_cuda(), name, " must be a CUDA tensor");
  TORCH_CHECK(t.scalar_type() == dt, name, " has the wrong dtype");
  TORCH_CHECK(t.is_contiguous(), name, " must be contiguous");
}

void check_rc(int rc, const char* what) {
  TORCH_CHECK(rc == FD3_OK, what, " failed (status ", rc, "): ", fd3_last_error());
}

// pos (N,3) float64 Angstrom on the device; species (N,) int32 compact ids on the device;
// cell (3,3) float64 Angstrom on the host (sizes the cell list); cell_dev the same cell on the
// device (copied from cell on the current stream when absent; a device cell that differs from
// the host cell makes every output NaN); work a uint8 device buffer of at least
// fd3_workspace_size bytes.
std::tuple<at::Tensor, at::Tensor, at::Tensor> energy_forces_stress_cuda(int64_t plan, const at::Tensor& pos,
                                                                         const at::Tensor& species,
                                                                         const at::Tensor& cell, double r_cut,
                                                                         const at::Tensor& work,
                                                                         const std::optional<at::Tensor>& cell_dev_in) {
  check_cuda(pos, at::kDouble, "pos");
  check_cuda(species, at::kInt, "species");
  check_cuda(work, at::kByte, "work");
  TORCH_CHECK(pos.dim() == 2 && pos.size(1) == 3, "pos must be (N, 3)");
  TORCH_CHECK(species.numel() == pos.size(0), "species must have N entries");
  TORCH_CHECK(!cell.is_cuda() && cell.scalar_type() == at::kDouble && cell.numel() == 9 && cell.is_contiguous(),
              "cell must be a contiguous (3, 3) float64 host tensor");
  const c10::cuda::CUDAGuard guard(pos.device());
  const int64_t n = pos.size(0);
  at::Tensor cell_dev = cell_dev_in.has_value() ? *cell_dev_in : cell.to(pos.device(), /*non_blocking=*/false);
  check_cuda(cell_dev, at::kDouble, "cell_dev");
  TORCH_CHECK(cell_dev.numel() == 9, "cell_dev must be (3, 3)");
  at::Tensor e = at::empty({}, pos.options());
  at::Tensor f = at::empty({n, 3}, pos.options());
  at::Tensor s = at::empty({3, 3}, pos.options());
  const cudaStream_t st = c10::cuda::getCurrentCUDAStream(pos.device().index()).stream();
  check_rc(fd3_energy_forces_stress(reinterpret_cast<fd3_plan*>(plan), n, pos.data_ptr<double>(),
                                    species.data_ptr<int32_t>(), cell.data_ptr<double>(),
                                    cell_dev.data_ptr<double>(), r_cut, work.data_ptr(), (size_t)work.numel(),
                                    e.data_ptr<double>(), f.data_ptr<double>(), s.data_ptr<double>(), st),
           "fd3_energy_forces_stress");
  return {e, f, s};
}

std::tuple<at::Tensor, at::Tensor, at::Tensor> energy_forces_stress_meta(int64_t, const at::Tensor& pos,
                                                                         const at::Tensor&, const at::Tensor&,
                                                                         double, const at::Tensor&,
                                                                         const std::optional<at::Tensor>&) {
  return {at::empty({}, pos.options()), at::empty({pos.size(0), 3}, pos.options()), at::empty({3, 3}, pos.options())};
}

// Module path: pos_bohr (N,3), cell_bohr (3,3), shifts_bohr (E,3) float64 on the device; src, dst
// (E,) int64 edge ends; returns (energy [Hartree], dE/dpos, dE/dshift, dE/dcell) with positions
// and shifts held fixed for the cell gradient (fd3_energy_edges).
std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor> energy_edges_cuda(
    int64_t plan, const at::Tensor& pos, const at::Tensor& species, const at::Tensor& cell, const at::Tensor& src,
    const at::Tensor& dst, const at::Tensor& shifts, bool need_grad, const at::Tensor& work) {
  check_cuda(pos, at::kDouble, "pos");
  check_cuda(species, at::kInt, "species");
  check_cuda(cell, at::kDouble, "cell");
  check_cuda(src, at::kLong, "src");
  check_cuda(dst, at::kLong, "dst");
  check_cuda(shifts, at::kDouble, "shifts");
  check_cuda(work, at::kByte, "work");
  TORCH_CHECK(pos.dim() == 2 && pos.size(1) == 3 && cell.numel() == 9, "pos must be (N, 3), cell (3, 3)");
  TORCH_CHECK(src.numel() == dst.numel() && shifts.numel() == 3 * src.numel(), "edge arrays disagree in length");
  const c10::cuda::CUDAGuard guard(pos.device());
  const int64_t n = pos.size(0), ne = src.numel();
  at::Tensor e = at::empty({}, pos.options());
  at::Tensor gp = at::empty({need_grad ? n : 0, 3}, pos.options());   // written in full by libfd3
  at::Tensor gs = at::empty({need_grad ? ne : 0, 3}, pos.options());
  at::Tensor gc = at::empty({need_grad ? 3 : 0, 3}, pos.options());
  const cudaStream_t st = c10::cuda::getCurrentCUDAStream(pos.device().index()).stream();
  check_rc(fd3_energy_edges(reinterpret_cast<fd3_plan*>(plan), n, pos.data_ptr<double>(), species.data_ptr<int32_t>(),
                            cell.data_ptr<double>(), ne, src.data_ptr<int64_t>(), dst.data_ptr<int64_t>(),
                            shifts.data_ptr<double>(), need_grad ? 1 : 0, work.data_ptr(), (size_t)work.numel(),
                            e.data_ptr<double>(), need_grad ? gp.data_ptr<double>() : nullptr,
                            need_grad ? gs.data_ptr<double>() : nullptr, need_grad ? gc.data_ptr<double>() : nullptr,
                            st),
           "fd3_energy_edges");
  return {e, gp, gs, gc};
}

std::tuple<at::Tensor, at::Tensor, at::Tensor, at::Tensor> energy_edges_meta(
    int64_t, const at::Tensor& pos, const at::Tensor&, const at::Tensor&, const at::Tensor& src, const at::Tensor&,
    const at::Tensor&, bool, const at::Tensor&) {
  return {at::empty({}, pos.options()), at::empty({pos.size(0), 3}, pos.options()),
          at::empty({src.numel(), 3}, pos.options()), at::empty({3, 3}, pos.options())};   // need_grad = true
}

}  // namespace

TORCH_LIBRARY(fd3, m) {
  m.def("energy_forces_stress(int plan, Tensor pos, Tensor species, Tensor cell, float r_cut, Tensor work, "
        "Tensor? cell_dev=None) -> (Tensor, Tensor, Tensor)");
  m.def("energy_edges(int plan, Tensor pos, Tensor species, Tensor cell, Tensor src, Tensor dst, Tensor shifts, "
        "bool need_grad, Tensor work) -> (Tensor, Tensor, Tensor, Tensor)");
}

TORCH_LIBRARY_IMPL(fd3, CUDA, m) {
  m.impl("energy_forces_stress", &energy_forces_stress_cuda);
  m.impl("energy_edges", &energy_edges_cuda);
}

TORCH_LIBRARY_IMPL(fd3, Meta, m) {
  m.impl("energy_forces_stress", &energy_forces_stress_meta);
  m.impl("energy_edges", &energy_edges_meta);
}
