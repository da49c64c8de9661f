// Drives the C++ world API (include/numi_world.hpp) the way a caller of the
// reference's MetalWorldContext would: one run() of a tree29 batch, and a
// pile batch advanced by initializeResidentState + submitResident.  Writes
// the tree's actions and both final states as raw float32 to the paths given
// on the command line.
#include "numi_world.hpp"

#include <cmath>
#include <cstdio>
#include <vector>

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s tree_out pile_out actions_out\n", argv[0]);
        return 2;
    }
    numi::WorldContext context;
    numi::WorldStepConfig config;  // 20 ms control, 4 substeps, 8 iterations
    // tree29: 4 envs x 6 control steps, deterministic PD targets.
    const std::size_t envs = 4, steps = 6, na = 29;
    std::vector<float> actions(steps * envs * na);
    for (std::size_t i = 0; i < actions.size(); ++i) actions[i] = 0.3f * std::sin(0.37f * static_cast<float>(i));
    numi::WorldBatch batch;
    batch.environment_count = envs;
    batch.control_step_count = steps;
    batch.actions = actions.data();
    batch.action_count = actions.size();
    numi::WorldResult tree;
    const numi::WorldDiagnostics d = context.run({MR_RUN_SOURCE_SYNTHETIC_TREE29, 11}, batch, config, tree);
    if (!d.succeeded || tree.final_q.size() != envs * tree.nq || tree.observations.size() != steps * envs * (tree.nq + tree.nv)) {
        std::fprintf(stderr, "tree run failed or incomplete\n");
        return 1;
    }
    // Pile: 3 envs, 10 control steps in two resident submissions.
    numi::WorldResidentState state;
    numi::WorldBatch pile;
    pile.environment_count = 3;
    pile.control_step_count = 4;
    numi::WorldResult first, second;
    context.initializeResidentState({MR_RUN_SOURCE_SYNTHETIC_PILE, 10}, pile, config, state, &first);
    pile.control_step_count = 6;
    const numi::WorldDiagnostics dp = context.submitResident({MR_RUN_SOURCE_SYNTHETIC_PILE, 10}, pile, config, state, &second);
    if (!dp.succeeded || second.final_scene_bodies.empty()) {
        std::fprintf(stderr, "pile submission failed\n");
        return 1;
    }
    std::FILE* f = std::fopen(argv[1], "wb");
    std::fwrite(tree.final_q.data(), sizeof(float), tree.final_q.size(), f);
    std::fclose(f);
    f = std::fopen(argv[2], "wb");
    std::fwrite(second.final_q.data(), sizeof(float), second.final_q.size(), f);
    std::fclose(f);
    f = std::fopen(argv[3], "wb");
    std::fwrite(actions.data(), sizeof(float), actions.size(), f);
    std::fclose(f);
    std::printf("ok tree nq=%u pile nq=%u\n", tree.nq, second.nq);
    return 0;
}
