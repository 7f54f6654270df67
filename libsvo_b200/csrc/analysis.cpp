// analysis.cpp -- host side of the analysis pass
// (RenderPassAnalyse::performAnalysePass, src/RenderPassAnalyse.cpp:218-356,
// and addNodeAndItsParentTreeletsToVisibleTreelets, :381-420).
//
// From the feedback records: every hit on a leaf whose sub-treelet is not
// resident names that treelet as newly visible (keeping the largest error
// seen for it); every hit names the treelet holding the hit node and all its
// ancestors as visible (largest error; the root treelet gets 99).  Both lists
// are ordered by error, largest first (the reference's multiset ordering:
// ties keep ascending gid order), and the new list is cut to the number of
// treelets that fit in 12 MB.
#include <algorithm>
#include <map>

#include "memory_manager.h"

namespace svo {

uint32_t TreeletMemoryManager::default_max_new_treelets() const {
  // static const unsigned maxTreeletsToPropergate = (12.0*1048576.0f)/treeletSize
  return (uint32_t)((12.0 * 1048576.0f) / (double)scene_.treelet_bytes);
}

int TreeletMemoryManager::analyse_feedback(const svo_feedback* fb, uint64_t n, uint32_t max_new,
                                           std::vector<std::pair<int32_t, float>>& out_new,
                                           std::vector<std::pair<int32_t, float>>& out_old) const {
  out_new.clear();
  out_old.clear();
  const uint64_t num_treelets = scene_.treelets.size();
  std::map<int32_t, float> visible_new, visible_old;
  for (uint64_t i = 0; i < n; ++i) {
    const svo_feedback& e = fb[i];
    if (e.node_id == 0) continue;
    if (e.sub_treelet_gid != 0) {
      // the reference rejects the whole pass on these (:257-263, > not >=)
      if (e.node_id < 0 || (uint64_t)(uint32_t)e.sub_treelet_gid > num_treelets) return SVO_ERR_RANGE;
      auto it = visible_new.find(e.sub_treelet_gid);
      if (it == visible_new.end())
        visible_new[e.sub_treelet_gid] = e.error;
      else if (e.error > it->second)
        it->second = e.error;
    }
    const uint32_t slot = (uint32_t)e.node_id / N_;
    if (slot > num_treelets || slot >= slots_.size()) return SVO_ERR_RANGE;  // :286-293
    const int32_t gid = slots_[slot].treelet_gid;
    if (gid < 0 || (uint64_t)gid > num_treelets) return SVO_ERR_RANGE;  // :297-304
    for (int32_t g = gid; g != 0;) {
      auto it = visible_old.find(g);
      if (it == visible_old.end())
        visible_old[g] = e.error;
      else if (e.error > it->second)
        it->second = e.error;
      if ((uint64_t)g >= num_treelets) return SVO_ERR_RANGE;
      g = scene_.treelets[g].parent_gid;
    }
    visible_old[0] = 99.0f;
  }
  for (const auto& kv : visible_new) out_new.emplace_back(kv.first, kv.second);
  for (const auto& kv : visible_old) out_old.emplace_back(kv.first, kv.second);
  auto by_error = [](const std::pair<int32_t, float>& a, const std::pair<int32_t, float>& b) {
    return a.second > b.second;
  };
  std::stable_sort(out_new.begin(), out_new.end(), by_error);
  std::stable_sort(out_old.begin(), out_old.end(), by_error);
  if (out_new.size() > max_new) out_new.resize(max_new);
  return SVO_OK;
}

}  // namespace svo
