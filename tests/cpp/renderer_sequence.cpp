// The call sequence of the reference's only caller of the builder
// (gpu-ray-traversal/src/rt/cuda/Renderer.cpp:164-228), compiled against
// include/bvhrt.hpp: SceneWrapper -> LBVHBuilder -> AgglomerativeTreeletOptimizer
// -> BVHTreeCollapser -> DeviceToHostCollapsedTree.  Prints the SAH values and
// the number of reachable leaves for the parity test to compare.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "bvhrt.hpp"

int main(int argc, char** argv) {
    const unsigned n = argc > 1 ? (unsigned)atoi(argv[1]) : 4096;
    std::vector<float> soup((size_t)n * 12);
    if (atr_gen_scene(ATR_SCENE_CLUSTERED, n, 2, soup.data()) != ATR_OK) return 2;
    float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {1.17549435e-38f, 1.17549435e-38f, 1.17549435e-38f};
    BVHRT::float4* verts = new BVHRT::float4[3 * (size_t)n];
    for (size_t i = 0; i < 3 * (size_t)n; ++i) {
        verts[i] = BVHRT::float4{soup[4 * i], soup[4 * i + 1], soup[4 * i + 2], 0.0f};
        const float c[3] = {soup[4 * i], soup[4 * i + 1], soup[4 * i + 2]};
        for (int k = 0; k < 3; ++k) {
            if (c[k] < mn[k]) mn[k] = c[k];
            if (c[k] > mx[k]) mx[k] = c[k];
        }
    }
    try {
        BVHRT::SceneWrapper* scene = new BVHRT::SceneWrapper(n, verts, BVHRT::float3{mn[0], mn[1], mn[2]},
                                                             BVHRT::float3{mx[0], mx[1], mx[2]});
        BVHRT::LBVHBuilder builder;
        BVHRT::BVHTree* tree = builder.BuildTree(scene);
        BVHRT::AgglomerativeTreeletOptimizer optimizer(9, 2);
        optimizer.Optimize(tree);
        BVHRT::BVHTreeInstanceManager manager;
        BVHRT::SoABVHTree* host = manager.DeviceToHostTree(tree);
        float sah = 0.0f;
        BVHRT::BVHTreeCollapser collapser;
        BVHRT::BVHCollapsedTree* collapsed = collapser.Collapse(tree, &sah);
        BVHRT::BVHCollapsedTree* hc = manager.DeviceToHostCollapsedTree(collapsed);
        int leaves = 0;
        std::vector<int> stack{hc->rootIndex};
        while (!stack.empty()) {
            const int x = stack.back();
            stack.pop_back();
            for (int ch : {hc->nodes.leftIndices[x], hc->nodes.rightIndices[x]}) {
                if (hc->nodes.dataIndices[ch] >= 0) ++leaves;
                else stack.push_back(ch);
            }
        }
        printf("tree_sah %.9g collapse_sah %.9g leaves %d\n", host->SAH(), sah, leaves);
        delete hc;
        delete host;
        manager.FreeDeviceCollapsedTree(collapsed);
        manager.FreeDeviceTree(tree);
        delete scene;
    } catch (const BVHRT::Error& e) {
        fprintf(stderr, "error %d: %s\n", e.status, e.what());
        return 1;
    }
    return 0;
}
