// graph_csr_mipmapped_device.cuh -- the device copy of a mipmapped graph
// (farkhor/KiTES kites/graph/graph_csr_mipmapped_device.cuh:14-84): the CSC,
// the block-level mipmap and two block-level frontier bitmaps, uploaded on
// the device's working stream.  Plain device buffers owned by the object
// (the engine's layout is not built for it: only the user-program pull of
// process() over a mipmapped graph reads these arrays).
//
// Additions beside the reference's members: `updateFlag` (the device flag
// process() clears and reads back) and `changedBlocks` (one bit per block,
// the blocks with an updated vertex in the current iteration).
#ifndef KITES_B200_GRAPH_CSR_MIPMAPPED_DEVICE_CUH_
#define KITES_B200_GRAPH_CSR_MIPMAPPED_DEVICE_CUH_

#include <chrono>
#include <iostream>

#include "../device/nv_gpu.cuh"
#include "../memory/device_buffer.cuh"
#include "../memory/mem_ops.cuh"
#include "graph_csr_mipmapped.hpp"

namespace kites {

template <class vT, class eT, class vIdxT = unsigned int>
class graph_csr_mipmapped_device : public graph_base {
  using eIdxT = vIdxT;

 public:
  int residing_device_id;

  device_buffer<vT> V;
  device_buffer<eIdxT> R;
  device_buffer<vIdxT> C;
  device_buffer<eT> E;
  host_pinned_buffer<unsigned int> updateFlagHost;

  unsigned int compressionRatio;
  unsigned int mipmapDim;
  device_bitmap mipmap;
  device_bitmap vBitmapEven;
  device_bitmap vBitmapOdd;
  device_buffer<unsigned int> compactionBuffer;
  device_buffer<unsigned int> updateFlag;
  device_bitmap changedBlocks;

  int getResidingDeviceID() const { return residing_device_id; }

  double accumulatedH2DCopyTime;

  graph_csr_mipmapped_device(graph_csr_mipmapped<vT, eT, vIdxT> &h, nv_gpu &dev)
      : residing_device_id{[&] { dev.setAsActive(); return dev.getDevIdx(); }()},
        V{h.V.size(), residing_device_id},
        R{h.R.size(), residing_device_id},
        C{h.C.size(), residing_device_id},
        E{h.E.size(), residing_device_id},
        updateFlagHost{h.updateFlag.size()},
        compressionRatio{h.compressionRatio},
        mipmapDim{h.mipmapDim},
        mipmap{h.mipmap.getnBits(), residing_device_id},
        vBitmapEven{h.vBitmap.getnBits(), residing_device_id},
        vBitmapOdd{h.vBitmap.getnBits(), residing_device_id},
        compactionBuffer{h.mipmapDim + 1u, residing_device_id},
        updateFlag{1, residing_device_id},
        changedBlocks{h.vBitmap.getnBits(), residing_device_id},
        accumulatedH2DCopyTime{0} {
    static_assert(sizeof(vIdxT) == 4, "vertex and edge indices are 32-bit");
    const auto t1 = std::chrono::steady_clock::now();
    stream &s = dev.getSsEven();
    copyMemOnStream(V, h.V, s);
    copyMemOnStream(R, h.R, s);
    copyMemOnStream(C, h.C, s);
    copyMemOnStream(E, h.E, s);
    copyMemOnStream(vBitmapEven, h.vBitmap, s);
    copyMemOnStream(mipmap, h.mipmap, s);
    s.sync();
    accumulatedH2DCopyTime =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t1).count();
    vBitmapOdd.reset(s);
    changedBlocks.reset(s);
    s.sync();
    set_num_edges(h.get_num_edges());
    set_num_vertices(h.get_num_vertices());
    std::cout << "H2D copies took " << accumulatedH2DCopyTime << " (ms) in total.\n";
  }
  graph_csr_mipmapped_device(const graph_csr_mipmapped_device &) = delete;
  graph_csr_mipmapped_device &operator=(const graph_csr_mipmapped_device &) = delete;
  graph_csr_mipmapped_device(graph_csr_mipmapped_device &&) noexcept = default;
};

// kites/graph/graph_csr_mipmapped_device.cuh:78-81
template <class vT, class eT, class vIdxT>
graph_csr_mipmapped_device<vT, eT, vIdxT> make_graph_csr_for_device(
    graph_csr_mipmapped<vT, eT, vIdxT> &h, nv_gpu &dev) {
  return graph_csr_mipmapped_device<vT, eT, vIdxT>(h, dev);
}

}  // namespace kites

#endif
