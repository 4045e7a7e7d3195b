// graph_csr_device.cuh -- the device graph of the kites:: API (farkhor/KiTES
// kites/graph/graph_csr_device.cuh:14-152).  Uploading goes through the C
// ABI (kites_graph_upload), which also builds the engine's B200 layout; the
// public members are non-owning views of the engine's arrays, so user code
// that reads devGrph.V (e.g. host_pinned_buffer<vT>(devGrph.V)) still works.
#ifndef KITES_B200_GRAPH_CSR_DEVICE_CUH_
#define KITES_B200_GRAPH_CSR_DEVICE_CUH_

#include <chrono>
#include <iostream>

#include "../../kites_b200.h"
#include "../device/nv_gpu.cuh"
#include "../memory/device_buffer.cuh"
#include "../memory/mem_ops.cuh"
#include "graph_csr.h"

namespace kites {

template <class vT, class eT, class vIdxT = unsigned int>
class graph_csr_device : public graph_base {
  using eIdxT = vIdxT;
  kites_graph *handle = nullptr;

 public:
  int residing_device_id = 0;
  device_buffer<vT> V;
  device_buffer<eIdxT> R;
  device_buffer<vIdxT> C;
  device_buffer<eT> E;
  device_bitmap vBitmapEven;
  device_bitmap vBitmapOdd;
  device_buffer<unsigned int> updateFlag;
  host_pinned_buffer<unsigned int> updateFlagHost;
  graph_property gProp = graph_property::directed;
  device_buffer<eIdxT> dir_R;
  device_buffer<vIdxT> dir_C;
  unsigned int vertexPerGroup = 1;
  // Device time (CUDA events around the loop) and iteration count of the
  // last kites::process call with user functions on this graph.
  float last_device_ms = 0.f;
  unsigned long long last_iterations = 0;

  int getResidingDeviceID() const { return residing_device_id; }
  unsigned int getVertexPerGroup() const { return vertexPerGroup; }
  kites_graph *engine_graph() const { return handle; }

  graph_csr_device() = default;
  graph_csr_device(graph_csr<vT, eT, vIdxT> &h, nv_gpu &dev)
      : residing_device_id{[&] { dev.setAsActive(); return dev.getDevIdx(); }()},
        updateFlagHost(1), gProp{h.gProp}, vertexPerGroup{h.getVertexPerGroup()} {
    static_assert(sizeof(vIdxT) == 4, "vertex and edge indices are 32-bit");
    auto t0 = std::chrono::steady_clock::now();
    kites_csc_view v{};
    v.n_vertices = h.get_num_vertices();
    v.n_edges = h.get_num_edges();
    v.row_offsets32 = reinterpret_cast<const uint32_t *>(h.R.get_ptr());
    v.col_indices = reinterpret_cast<const uint32_t *>(h.C.get_ptr());
    v.edge_values = h.E.get_ptr();
    v.edge_value_size = sizeof(eT);
    v.vertex_value_size = sizeof(vT);
    v.vertex_values = h.V.get_ptr();
    v.vertex_per_group = h.getVertexPerGroup();
    v.directed = h.gProp == graph_property::directed ? 1 : 0;
    v.frontier_bits = h.vBitmap.get_ptr();
    v.frontier_nbits = h.vBitmap.getnBits();
    if (v.directed && h.dir_R.size()) {
      v.n_out_rows = h.dir_R.size() - 1;
      v.out_row_offsets32 = reinterpret_cast<const uint32_t *>(h.dir_R.get_ptr());
      v.out_col_indices = reinterpret_cast<const uint32_t *>(h.dir_C.get_ptr());
      v.n_out_edges = h.dir_C.size();
    }
    KITESErrorCheck(kites_graph_upload(dev.engine(), &v, &handle));
    bind_views();
    set_num_vertices(h.get_num_vertices());
    set_num_edges(h.get_num_edges());
    const double ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "H2D copies took " << ms << " (ms) in total.\n";
  }
  graph_csr_device(const graph_csr_device &) = delete;
  graph_csr_device &operator=(const graph_csr_device &) = delete;
  graph_csr_device(graph_csr_device &&o) noexcept
      : graph_base(o), handle{o.handle}, residing_device_id{o.residing_device_id},
        V(std::move(o.V)), R(std::move(o.R)), C(std::move(o.C)), E(std::move(o.E)),
        vBitmapEven(std::move(o.vBitmapEven)), vBitmapOdd(std::move(o.vBitmapOdd)),
        updateFlag(std::move(o.updateFlag)), updateFlagHost(std::move(o.updateFlagHost)),
        gProp{o.gProp}, dir_R(std::move(o.dir_R)), dir_C(std::move(o.dir_C)),
        vertexPerGroup{o.vertexPerGroup} {
    o.handle = nullptr;
  }
  ~graph_csr_device() {
    if (handle) kites_graph_destroy(handle);
  }

 private:
  void bind_views() {
    kites_device_view dv{};
    KITESErrorCheck(kites_graph_device_view(handle, &dv));
    if (dv.offsets64) throw std::runtime_error("graph needs 64-bit offsets; kites::graph_csr uses 32-bit");
    const int d = residing_device_id;
    V = device_buffer<vT>::view(static_cast<vT *>(dv.V), get_n(dv), d);
    R = device_buffer<eIdxT>::view((eIdxT *)dv.R, dv.n_vertices + 1, d);
    C = device_buffer<vIdxT>::view((vIdxT *)dv.C, dv.n_edges, d);
    E = device_buffer<eT>::view(static_cast<eT *>(dv.E), dv.E ? dv.n_edges : 0, d);
    vBitmapEven = device_bitmap(device_buffer<unsigned int>::view(dv.frontier[0], (dv.nbits + 31) / 32, d), dv.nbits);
    vBitmapOdd = device_bitmap(device_buffer<unsigned int>::view(dv.frontier[1], (dv.nbits + 31) / 32, d), dv.nbits);
    updateFlag = device_buffer<unsigned int>::view(dv.update_flag, 1, d);
  }
  static std::size_t get_n(const kites_device_view &dv) { return dv.n_vertices; }
};

// kites/graph/graph_csr_device.cuh:146-152
template <class vT, class eT, class vIdxT>
graph_csr_device<vT, eT, vIdxT> make_graph_csr_for_device(graph_csr<vT, eT, vIdxT> &h, nv_gpu &dev) {
  return graph_csr_device<vT, eT, vIdxT>(h, dev);
}

}  // namespace kites

#endif
