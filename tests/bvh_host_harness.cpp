// Test harness for the host BVH builder (cupbr_b200/csrc/bvh_build.cpp):
// reads n primitive boxes (6 float32 each) from argv[1], builds one tree
// with max_leaf argv[3], writes to argv[2]:
//   uint32 n_nodes, leaves, max_depth; float64 sah;
//   n_nodes * 32 float32 node words; n uint32 leaf order (perm).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bvh_build.hpp"

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s boxes.bin out.bin max_leaf\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    std::vector<cupbr_b200::PrimBox> boxes[3];
    cupbr_b200::PrimBox b;
    while (std::fread(&b, sizeof b, 1, f) == 1) boxes[0].push_back(b);
    std::fclose(f);
    cupbr_b200::BvhBuildParams p;
    p.max_leaf = std::atoi(argv[3]);
    p.device = false;
    const uint32_t offs[3] = {0u, (uint32_t)boxes[0].size(), (uint32_t)boxes[0].size()};
    std::vector<uint32_t> perm[3];
    cupbr_b200::FlatBvh out;
    cupbr_b200::build_bvh(boxes, 3, offs, p, perm, out);
    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 4;
    const uint32_t hdr[3] = {(uint32_t)(out.nodes.size() / (4 * cupbr_b200::BVH_NODE_F4)), out.stats.leaves,
                             out.stats.max_depth};
    std::fwrite(hdr, sizeof hdr, 1, o);
    std::fwrite(&out.stats.sah_cost, sizeof(double), 1, o);
    std::fwrite(out.nodes.data(), sizeof(float), out.nodes.size(), o);
    std::fwrite(perm[0].data(), sizeof(uint32_t), perm[0].size(), o);
    std::fclose(o);
    return 0;
}
