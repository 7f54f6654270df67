// frame_loop.cpp -- the reference app's init() / frameStep() written against
// the C++ drop-in class (include/libsvo_b200.hpp), with the method names a
// TreeletMemoryManagerCl user already calls (raycast_serialized_opencl.cpp:
// 315-324 and 684-747).
//
//   frame_loop_cpp <svo_path_base> <incore_bytes> <frames> <params.bin> <out_base>
//
// Per frame: performAnalysePass (analysis, updateClientSideIncoreBuffer,
// updateDeviceMemory), then on the last frame renderToBuffer into a device
// image read back to the host.  Before the loop, a first manager over the
// same file exercises the manual slot API (insert, getSlots,
// freeIncorePosition, remove, reset) and checks its bookkeeping; the loop
// runs on a second, fresh one.  Writes <out_base>.rgba, .nodes and .attribs
// like frame_loop.c.  Exit status 0 on success.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <vector>

#include "libsvo_b200.hpp"

static bool write_file(const std::string& path, const void* data, size_t bytes) {
  std::ofstream f(path, std::ios::binary);
  f.write(static_cast<const char*>(data), (std::streamsize)bytes);
  return (bool)f;
}

static int check(bool ok, const char* what) {
  if (!ok) std::cerr << what << " failed: " << svo_last_error() << "\n";
  return ok ? 0 : 1;
}

int main(int argc, char** argv) {
  if (argc != 6) {
    std::cerr << "usage: frame_loop_cpp svo_path_base incore_bytes frames params.bin out_base\n";
    return 2;
  }
  const uint64_t incore = std::strtoull(argv[2], nullptr, 10);
  const long n = std::strtol(argv[3], nullptr, 10);
  if (n <= 0) return 2;
  std::vector<svo_frame_params> frames((size_t)n);
  {
    std::ifstream f(argv[4], std::ios::binary);
    f.read(reinterpret_cast<char*>(frames.data()), (std::streamsize)(n * sizeof(svo_frame_params)));
    if (!f) return 3;
  }
  try {
    {  // the manual slot API on a first manager
      svo::TreeletMemoryManagerCuda mm(argv[1], incore);
      mm.initDeviceBuffer();
      const unsigned slots = (unsigned)mm.getSlots().size();
      if (slots == 0 || mm.getNumNodesPerTreelet() * 8u != mm.getTreeletSizeInByte()) return 4;

      // the manual slot API: insert the root's first children, free one
      // position, remove, reset back to the root alone
      int inserted = 0;
      for (int g = 1; g < (int)mm.getNumTreelets() && inserted < 3; ++g) {
        svo::TreeletMemoryManagerCuda::SlotInfo tve(g, 1, 0.5f);
        if (mm.insertTreeletIntoIncoreBuffer(tve)) ++inserted;
      }
      if (inserted > 0) {
        int resident = 0;
        for (const auto& s : mm.getSlots()) resident += s._treeletGid >= 0;
        if (resident != inserted + 1) return 5;  // + the root treelet in slot 0
        if (mm.getIncoreSlotsToUpload().empty()) return 6;
        if (check(mm.updateDeviceMemory(), "updateDeviceMemory")) return 7;
        // freeIncorePosition evicts only treelets marked invisible: none here
        if (mm.freeIncorePosition()) return 8;
        const int gid = mm.getSlots()[1]._treeletGid;
        if (gid > 0 && check(mm.removeTreeletFromIncoreBuffer(gid), "removeTreeletFromIncoreBuffer")) return 9;
        if (gid > 0 && mm.getTreeletSlotGid(gid) != -1) return 10;
      }
      if (check(mm.resetIncoreBuffer(), "resetIncoreBuffer")) return 11;
      if (mm.getNumFreeIncoreSlots() != slots - 1) return 12;
      if (check(mm.updateDeviceMemory(), "updateDeviceMemory")) return 13;
    }

    // init(): the manager over the treelet file, then the device buffer
    svo::TreeletMemoryManagerCuda mm(argv[1], incore);
    mm.initDeviceBuffer();
    const unsigned slots = (unsigned)mm.getSlots().size();
    // frameStep(): analysis pass with paging, then the frame
    const svo_frame_params& last = frames.back();
    std::vector<uint32_t> rgba((size_t)last.width * last.height);
    uint32_t placed_total = 0;
    for (long i = 0; i < n; ++i) {
      placed_total += mm.performAnalysePass(frames[(size_t)i], 1);
      if (i == n - 1 && check(mm.renderToHostBuffer(last, rgba.data()), "renderToHostBuffer")) return 14;
    }
    const svo_stats st = mm.sync();
    const std::vector<svo_node> nodes = mm.getIncoreBuffer();
    const std::vector<svo_attrib> attribs = mm.getAttributeIncoreBuffer();
    const std::string out = argv[5];
    if (!write_file(out + ".rgba", rgba.data(), rgba.size() * 4) ||
        !write_file(out + ".nodes", nodes.data(), nodes.size() * sizeof(svo_node)) ||
        !write_file(out + ".attribs", attribs.data(), attribs.size() * sizeof(svo_attrib)))
      return 15;
    std::printf("placed %u resident %u of %u capped %u bounds %u\n", placed_total,
                slots - mm.getNumFreeIncoreSlots(), mm.getNumTreelets(), st.capped_rays,
                st.bounds_errors);
  } catch (const svo::Error& e) {
    std::cerr << e.what() << "\n";
    return e.status() < 0 ? -e.status() : 1;
  }
  return 0;
}
