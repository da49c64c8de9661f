// Continuous-batching rollout server behind the C ABI (include/numi_b200.h,
// mr_create_server ... mr_server_release).
//
// Each world source (7-DoF chain, 29-DoF tree, pile) owns a pool of resident
// environment slots on the device: state, manifolds and friction live there
// for the whole life of a request.  Requests queue on submit; every tick
// admits waiting requests into free slots (first-come first-served with
// backfill, against an HBM budget), then advances every admitted request by
// one control step -- all requests of a pool packed into one launch of the
// control-step kernel through a work-item -> slot index and per-item action
// rows, the pools on their own streams so their work overlaps on the
// device -- and retires the requests whose horizon is complete, copying
// their final state out and freeing their slots.  An environment's
// trajectory depends only on its request (model, seed, index, actions), never
// on the slot it occupies or on the other requests in the launch.
#include "numi_b200.h"
#include "runtime.h"

#include <chrono>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <vector>

namespace {

using numi::rt::check;
using numi::rt::DeviceBuffer;
using numi::rt::guarded;
using numi::rt::PinnedBuffer;

// rows[i] (width floats) -> slots dst[index[i]]; zero when src is null.
__global__ void scatter_rows_kernel(float* __restrict__ dst, const float* __restrict__ src, const std::int32_t* __restrict__ index,
                                    int rows, int width) {
    const int total = rows * width;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int r = k / width, c = k - r * width;
        dst[static_cast<size_t>(index[r]) * width + c] = src != nullptr ? src[k] : 0.0f;
    }
}

// Staged reset rows [i][nq + nv + 1] -> q, v and friction of slot index[i].
__global__ void scatter_staged_kernel(float* __restrict__ q, float* __restrict__ v, float* __restrict__ friction,
                                      const float* __restrict__ stage, const std::int32_t* __restrict__ index, int rows, int nq,
                                      int nv) {
    const int width = nq + nv + 1;
    const int total = rows * width;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int r = k / width, c = k - r * width;
        const size_t slot = static_cast<size_t>(index[r]);
        const float x = stage[k];
        if (c < nq) q[slot * nq + c] = x;
        else if (c < nq + nv) v[slot * nv + (c - nq)] = x;
        else friction[slot] = x;
    }
}

// slots src[index[i]] -> rows dst[i] (width floats).
__global__ void gather_rows_kernel(float* __restrict__ dst, const float* __restrict__ src, const std::int32_t* __restrict__ index,
                                   int rows, int width) {
    const int total = rows * width;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < total; k += gridDim.x * blockDim.x) {
        const int r = k / width, c = k - r * width;
        dst[k] = src[static_cast<size_t>(index[r]) * width + c];
    }
}

int grid_for(int total) { return std::max(1, std::min(1184, (total + 255) / 256)); }

constexpr std::size_t kPoolCount = 3;  // chain, tree, pile
// Longest horizon the action arena is sized for (longer requests still fit
// when the arena has room: it is a shared pool, not per request).
constexpr std::size_t kArenaHorizon = 500;

double now_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// First-fit allocator over a preallocated device arena (offsets in floats):
// admission and retirement move ranges, never device memory.
struct Arena {
    std::map<std::size_t, std::size_t> free_ranges;  // offset -> length
    void reset(std::size_t words) {
        free_ranges.clear();
        if (words) free_ranges[0] = words;
    }
    bool take(std::size_t words, std::size_t& at) {
        if (words == 0) {
            at = 0;
            return true;
        }
        for (auto it = free_ranges.begin(); it != free_ranges.end(); ++it) {
            if (it->second < words) continue;
            at = it->first;
            const std::size_t rest = it->second - words;
            free_ranges.erase(it);
            if (rest) free_ranges[at + words] = rest;
            return true;
        }
        return false;
    }
    void give(std::size_t at, std::size_t words) {
        if (words == 0) return;
        auto next = free_ranges.lower_bound(at);
        if (next != free_ranges.end() && at + words == next->first) {
            words += next->second;
            next = free_ranges.erase(next);
        }
        if (next != free_ranges.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == at) {
                prev->second += words;
                return;
            }
        }
        free_ranges[at] = words;
    }
};

struct Request {
    std::uint64_t id = 0;
    std::uint32_t source = 0;
    std::uint32_t envs = 0;
    std::uint32_t horizon = 0;
    std::uint64_t seed = 0;
    std::vector<float> host_actions;  // [horizon][envs][actions], until admitted
    std::size_t arena_at = 0, arena_words = 0;  // actions in the pool's arena
    std::vector<std::int32_t> slots;
    std::uint32_t step = 0;
    std::uint32_t failed_env_steps = 0;
    std::uint32_t first_failure_status = 0;
    double t_submit = 0.0, t_admit = 0.0, t_finish = 0.0;
    std::vector<float> final_q, final_v;
    std::size_t out_at = 0;  // rows in the pool's result staging while retiring
};

struct Pool {
    std::uint32_t source = 0;
    numi::CompiledModel model;
    numi::rt::KernelPlan plan;
    bool scene = false;              // pile world: free-body kernel
    numi::SceneModel smodel{};
    std::uint32_t capacity = 0;
    std::uint32_t nq = 0, nv = 0, na = 0, manifold_words = 0, workspace_words = 0;
    cudaStream_t stream = nullptr;
    DeviceBuffer<numi::DeviceModel> d_model;
    DeviceBuffer<numi::SceneModel> d_smodel;
    DeviceBuffer<float> d_q, d_v, d_manifolds, d_friction, d_workspace;
    DeviceBuffer<std::uint32_t> d_mcount;  // live manifolds per slot (piles)
    // Preallocated per pool: request actions, the per-step item -> slot
    // index and action rows of a tick, statuses, reset-state staging of the
    // tick's admissions and result staging of its retirements.
    DeviceBuffer<float> d_arena;
    Arena arena;
    DeviceBuffer<std::int32_t> d_index, d_admit_slots, d_out_slots;
    DeviceBuffer<const float*> d_rows;
    DeviceBuffer<std::uint32_t> d_status, d_stats;
    DeviceBuffer<float> d_stage, d_out;
    PinnedBuffer<std::int32_t> h_index, h_admit_slots, h_out_slots;
    PinnedBuffer<const float*> h_rows;
    PinnedBuffer<std::uint32_t> h_status;
    PinnedBuffer<float> h_stage, h_out;
    std::vector<std::int32_t> free_slots;  // kept sorted descending; back() is the lowest
    std::vector<Request*> active;          // admission order
    std::vector<Request*> admitted;        // admitted in this tick (reset states staged)
    std::vector<std::uint32_t> step_items; // items of each control step of the tick
    std::uint32_t tick_env_steps = 0;

    std::size_t slot_bytes() const {
        return (static_cast<std::size_t>(nq) + nv + manifold_words + workspace_words + 1 + (scene ? 1 : 0)) * sizeof(float);
    }
    ~Pool() {
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace

struct MRServerHandle {
    MRServerConfigC config{};
    float h = 0.0f;
    std::uint32_t steps_per_tick = 1;
    std::map<std::uint32_t, std::unique_ptr<Pool>> pools;
    std::deque<std::unique_ptr<Request>> pending;
    std::vector<std::unique_ptr<Request>> running;
    std::map<std::uint64_t, std::unique_ptr<Request>> completed;
    std::vector<std::uint64_t> unreported;
    std::uint64_t next_id = 1;
    std::size_t budget_used = 0;
    std::uint64_t completed_env_steps = 0;

    Pool& pool(std::uint32_t source) {
        auto it = pools.find(source);
        if (it == pools.end()) throw std::invalid_argument("unsupported request source " + std::to_string(source));
        return *it->second;
    }

    void add_pool(std::uint32_t source) {
        auto p = std::make_unique<Pool>();
        p->source = source;
        p->model = source == MR_RUN_SOURCE_SYNTHETIC_CHAIN7   ? numi::build_chain7(config.model_seed)
                   : source == MR_RUN_SOURCE_SYNTHETIC_TREE29 ? numi::build_tree29(config.model_seed)
                                                              : numi::build_pile(config.model_seed);
        p->scene = p->model.scene;
        p->nq = p->model.world.nq;
        p->nv = p->model.world.nv;
        p->na = p->model.world.action_count;
        if (p->scene) {
            p->smodel = numi::rt::pack_scene(p->model, h);
            check(numi::configure_scene_step_kernel(), "scene kernel attributes");
            p->manifold_words = static_cast<std::uint32_t>(numi::kSceneManifolds * numi::kSceneSlotWords);
            p->workspace_words = static_cast<std::uint32_t>(numi::scene_workspace_words());
        } else {
            numi::rt::make_plan(p->model, h, p->plan);
            p->manifold_words = p->model.world.pair_count * numi::kManifoldWords;
        }
        // Slots: the configured maximum, bounded by this pool's share of the
        // HBM budget (half of it split across the pools); the action arena
        // takes the pool's share of the other half, at most what a full
        // pool of kArenaHorizon-step requests needs.
        const std::size_t share = config.hbm_budget_bytes / (2 * kPoolCount);
        p->capacity = static_cast<std::uint32_t>(std::min<std::size_t>(config.max_envs_per_source, share / p->slot_bytes()));
        if (p->capacity == 0) throw std::invalid_argument("the HBM budget holds no environment of source " + std::to_string(source));
        const std::size_t cap = p->capacity;
        const std::size_t arena_words =
            std::min<std::size_t>(share / sizeof(float), cap * kArenaHorizon * static_cast<std::size_t>(p->na));
        budget_used += cap * p->slot_bytes() + arena_words * sizeof(float);
        check(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream");
        if (p->scene) {
            p->d_smodel.resize(1);
            check(cudaMemcpy(p->d_smodel.ptr, &p->smodel, sizeof(numi::SceneModel), cudaMemcpyHostToDevice), "upload scene model");
        } else {
            p->d_model.resize(1);
            check(cudaMemcpy(p->d_model.ptr, &p->plan.dmodel, sizeof(numi::DeviceModel), cudaMemcpyHostToDevice), "upload model");
        }
        p->d_q.resize(cap * p->nq);
        p->d_v.resize(cap * p->nv);
        if (p->manifold_words) p->d_manifolds.resize(cap * p->manifold_words);
        if (p->scene) {
            p->d_mcount.resize(cap);
            p->d_workspace.resize(cap * p->workspace_words);
        }
        p->d_friction.resize(cap);
        p->d_arena.resize(std::max<std::size_t>(arena_words, 1));
        p->arena.reset(arena_words);
        const std::size_t items = cap * steps_per_tick;
        p->d_index.resize(items);
        p->d_rows.resize(items);
        p->d_status.resize(items);
        p->d_stats.resize(numi::kStatCount);
        p->d_admit_slots.resize(cap);
        p->d_out_slots.resize(cap);
        const std::size_t row = static_cast<std::size_t>(p->nq) + p->nv + 1;
        p->d_stage.resize(cap * row);
        p->d_out.resize(cap * (p->nq + p->nv));
        p->h_index.resize(items);
        p->h_rows.resize(items);
        p->h_status.resize(items);
        p->h_admit_slots.resize(cap);
        p->h_out_slots.resize(cap);
        p->h_stage.resize(cap * row);
        p->h_out.resize(cap * (p->nq + p->nv));
        for (std::int32_t s = static_cast<std::int32_t>(cap) - 1; s >= 0; --s) p->free_slots.push_back(s);
        pools[source] = std::move(p);
    }

    // Reserves slots and arena room; stages the request's reset states and
    // enqueues its actions (no device allocation, no synchronisation).
    bool try_admit(Request& r) {
        Pool& p = pool(r.source);
        if (p.free_slots.size() < r.envs) return false;
        const std::size_t words = r.host_actions.size();
        std::size_t at = 0;
        if (!p.arena.take(words, at)) return false;
        r.arena_at = at;
        r.arena_words = words;
        for (std::uint32_t e = 0; e < r.envs; ++e) {
            r.slots.push_back(p.free_slots.back());
            p.free_slots.pop_back();
        }
        if (words)  // from pageable memory: the span is consumed when the call returns
            check(cudaMemcpyAsync(p.d_arena.ptr + at, r.host_actions.data(), words * sizeof(float), cudaMemcpyHostToDevice, p.stream),
                  "request actions H2D");
        r.host_actions.clear();
        r.host_actions.shrink_to_fit();
        // Reset states packed after the tick's earlier admissions:
        // [env][nq + nv + 1 (friction)].
        std::size_t staged = 0;
        for (Request* a : p.admitted) staged += a->envs;
        const std::size_t row = static_cast<std::size_t>(p.nq) + p.nv + 1;
        for (std::uint32_t e = 0; e < r.envs; ++e) {
            float* dst = p.h_stage.ptr + (staged + e) * row;
            numi::sample_reset_state(p.model, r.seed, e, dst, dst + p.nq, dst + p.nq + p.nv);
            p.h_admit_slots.ptr[staged + e] = r.slots[e];
        }
        r.t_admit = now_seconds();
        p.admitted.push_back(&r);
        p.active.push_back(&r);
        return true;
    }

    // The tick's admissions of a pool: one staging copy and one scatter per
    // field into their slots.
    void scatter_admissions(Pool& p) {
        std::size_t n = 0;
        for (Request* a : p.admitted) n += a->envs;
        if (n == 0) return;
        const std::size_t row = static_cast<std::size_t>(p.nq) + p.nv + 1;
        check(cudaMemcpyAsync(p.d_stage.ptr, p.h_stage.ptr, n * row * sizeof(float), cudaMemcpyHostToDevice, p.stream), "reset H2D");
        check(cudaMemcpyAsync(p.d_admit_slots.ptr, p.h_admit_slots.ptr, n * sizeof(std::int32_t), cudaMemcpyHostToDevice, p.stream),
              "slots H2D");
        const int envs = static_cast<int>(n);
        scatter_staged_kernel<<<grid_for(envs * static_cast<int>(row)), 256, 0, p.stream>>>(
            p.d_q.ptr, p.d_v.ptr, p.d_friction.ptr, p.d_stage.ptr, p.d_admit_slots.ptr, envs, static_cast<int>(p.nq),
            static_cast<int>(p.nv));
        if (p.manifold_words)
            scatter_rows_kernel<<<grid_for(envs * static_cast<int>(p.manifold_words)), 256, 0, p.stream>>>(
                p.d_manifolds.ptr, nullptr, p.d_admit_slots.ptr, envs, static_cast<int>(p.manifold_words));
        if (p.scene)  // no live manifolds (zero words are a zero count)
            scatter_rows_kernel<<<grid_for(envs), 256, 0, p.stream>>>(reinterpret_cast<float*>(p.d_mcount.ptr), nullptr,
                                                                      p.d_admit_slots.ptr, envs, 1);
        check(cudaGetLastError(), "admission scatter");
        p.admitted.clear();
    }

    // Up to steps_per_tick control steps of every active request of the
    // pool (a request stops at its horizon), one launch per step.
    void launch(Pool& p) {
        p.step_items.assign(steps_per_tick, 0);
        p.tick_env_steps = 0;
        if (p.active.empty()) return;
        std::uint32_t n = 0;
        for (std::uint32_t j = 0; j < steps_per_tick; ++j) {
            std::uint32_t items = 0;
            for (Request* r : p.active) {
                if (r->step + j >= r->horizon) continue;
                const float* base = p.d_arena.ptr + r->arena_at + static_cast<std::size_t>(r->step + j) * r->envs * p.na;
                for (std::uint32_t e = 0; e < r->envs; ++e) {
                    p.h_index.ptr[n] = r->slots[e];
                    p.h_rows.ptr[n] = base + static_cast<std::size_t>(e) * p.na;
                    ++n;
                    ++items;
                }
            }
            p.step_items[j] = items;
        }
        p.tick_env_steps = n;
        if (n == 0) return;
        check(cudaMemcpyAsync(p.d_index.ptr, p.h_index.ptr, n * sizeof(std::int32_t), cudaMemcpyHostToDevice, p.stream), "index H2D");
        check(cudaMemcpyAsync(p.d_rows.ptr, p.h_rows.ptr, n * sizeof(const float*), cudaMemcpyHostToDevice, p.stream), "rows H2D");
        check(cudaMemsetAsync(p.d_stats.ptr, 0, numi::kStatCount * sizeof(std::uint32_t), p.stream), "clear stats");
        std::uint32_t off = 0;
        for (std::uint32_t j = 0; j < steps_per_tick; ++j) {
            const std::uint32_t items = p.step_items[j];
            if (items == 0) break;
            if (p.scene) {
                numi::SceneParams sp{};
                sp.model = p.d_smodel.ptr;
                sp.q = p.d_q.ptr;
                sp.v = p.d_v.ptr;
                sp.manifolds = p.d_manifolds.ptr;
                sp.manifold_count = p.d_mcount.ptr;
                sp.reset_q = p.d_q.ptr;  // no resets inside a request
                sp.reset_v = p.d_v.ptr;
                sp.friction_scale = p.d_friction.ptr;
                sp.env_index = p.d_index.ptr + off;
                sp.status_codes = p.d_status.ptr + off;
                sp.stats = p.d_stats.ptr;
                sp.workspace = p.d_workspace.ptr;
                sp.env_count = static_cast<int>(items);
                sp.substeps = static_cast<int>(config.physics_substeps);
                sp.velocity_iterations = static_cast<int>(config.velocity_iterations);
                sp.final_velocity_iterations = static_cast<int>(config.final_velocity_iterations);
                sp.support_mapped = p.smodel.support_mapped;
                check(numi::launch_scene_step(sp, p.stream), "scene step launch");
            } else {
                numi::StepParams sp{};
                sp.model = p.d_model.ptr;
                sp.q = p.d_q.ptr;
                sp.v = p.d_v.ptr;
                sp.manifolds = p.d_manifolds.ptr;
                sp.reset_q = p.d_q.ptr;  // no resets inside a request
                sp.reset_v = p.d_v.ptr;
                sp.friction_scale = p.d_friction.ptr;
                sp.actions = nullptr;
                sp.action_rows = p.d_rows.ptr + off;
                sp.env_index = p.d_index.ptr + off;
                sp.status_codes = p.d_status.ptr + off;
                sp.stats = p.d_stats.ptr;
                sp.env_count = static_cast<int>(items);
                sp.substeps = static_cast<int>(config.physics_substeps);
                sp.velocity_iterations = static_cast<int>(config.velocity_iterations);
                sp.final_velocity_iterations = static_cast<int>(config.final_velocity_iterations);
                check(numi::launch_control_step(sp, p.plan.layout[0], p.plan.contact, MR_PRECISION_FP32, false, p.plan.warps_per_block[0][0],
                                                p.stream),
                      "control step launch");
            }
            off += items;
        }
        check(cudaMemcpyAsync(p.h_status.ptr, p.d_status.ptr, n * sizeof(std::uint32_t), cudaMemcpyDeviceToHost, p.stream),
              "status D2H");
        // Final states of the requests this tick completes, gathered into the
        // result staging and copied out with the statuses.
        std::size_t rows = 0;
        for (Request* r : p.active) {
            if (r->step + steps_per_tick < r->horizon) continue;
            r->out_at = rows;
            for (std::uint32_t e = 0; e < r->envs; ++e) p.h_out_slots.ptr[rows + e] = r->slots[e];
            rows += r->envs;
        }
        if (rows) {
            const int m = static_cast<int>(rows);
            check(cudaMemcpyAsync(p.d_out_slots.ptr, p.h_out_slots.ptr, rows * sizeof(std::int32_t), cudaMemcpyHostToDevice, p.stream),
                  "result slots H2D");
            gather_rows_kernel<<<grid_for(m * static_cast<int>(p.nq)), 256, 0, p.stream>>>(p.d_out.ptr, p.d_q.ptr, p.d_out_slots.ptr, m,
                                                                                          static_cast<int>(p.nq));
            gather_rows_kernel<<<grid_for(m * static_cast<int>(p.nv)), 256, 0, p.stream>>>(
                p.d_out.ptr + rows * p.nq, p.d_v.ptr, p.d_out_slots.ptr, m, static_cast<int>(p.nv));
            check(cudaGetLastError(), "gather");
            check(cudaMemcpyAsync(p.h_out.ptr, p.d_out.ptr, rows * (p.nq + p.nv) * sizeof(float), cudaMemcpyDeviceToHost, p.stream),
                  "results D2H");
        }
    }

    void retire(Pool& p, double t_now) {
        std::vector<std::uint32_t> off(steps_per_tick, 0);
        for (std::uint32_t j = 1; j < steps_per_tick; ++j) off[j] = off[j - 1] + p.step_items[j - 1];
        std::vector<std::uint32_t> seen(steps_per_tick, 0);
        std::vector<Request*> still;
        std::size_t rows = 0;
        for (Request* r : p.active) rows += (r->step + steps_per_tick >= r->horizon) ? r->envs : 0;
        for (Request* r : p.active) {
            const std::uint32_t steps = std::min(steps_per_tick, r->horizon - r->step);
            for (std::uint32_t j = 0; j < steps; ++j) {
                for (std::uint32_t e = 0; e < r->envs; ++e) {
                    const std::uint32_t code = p.h_status.ptr[off[j] + seen[j] + e];
                    if (code != MR_STEP_SUCCESS) {
                        if (r->failed_env_steps == 0) r->first_failure_status = code;
                        ++r->failed_env_steps;
                    }
                }
                seen[j] += r->envs;
            }
            r->step += steps;
            completed_env_steps += static_cast<std::uint64_t>(r->envs) * steps;
            if (r->step < r->horizon) {
                still.push_back(r);
                continue;
            }
            r->final_q.assign(p.h_out.ptr + r->out_at * p.nq, p.h_out.ptr + (r->out_at + r->envs) * p.nq);
            r->final_v.assign(p.h_out.ptr + rows * p.nq + r->out_at * p.nv, p.h_out.ptr + rows * p.nq + (r->out_at + r->envs) * p.nv);
            r->t_finish = t_now;
            for (std::int32_t s : r->slots) p.free_slots.push_back(s);
            std::sort(p.free_slots.begin(), p.free_slots.end(), std::greater<std::int32_t>());
            p.arena.give(r->arena_at, r->arena_words);
            for (auto it = running.begin(); it != running.end(); ++it)
                if (it->get() == r) {
                    unreported.push_back(r->id);
                    completed[r->id] = std::move(*it);
                    running.erase(it);
                    break;
                }
        }
        p.active.swap(still);
    }
};

extern "C" {

MR_API MRServerHandle* mr_create_server(const MRServerConfigC* config) {
    std::unique_ptr<MRServerHandle> server;
    const int rc = guarded([&] {
        if (config == nullptr) throw std::invalid_argument("config is null");
        if (config->physics_substeps == 0 || config->physics_substeps > MR_B200_MAX_SUBSTEPS)
            throw std::invalid_argument("physics_substeps must be in [1, 64]");
        if (!(config->control_timestep_seconds > 0.0f)) throw std::invalid_argument("control_timestep_seconds must be positive");
        if (config->velocity_iterations == 0 && config->final_velocity_iterations == 0)
            throw std::invalid_argument("contact worlds need at least one velocity iteration");
        if (config->max_envs_per_source == 0) throw std::invalid_argument("max_envs_per_source must be positive");
        server = std::make_unique<MRServerHandle>();
        server->config = *config;
        server->h = config->control_timestep_seconds / static_cast<float>(config->physics_substeps);
        server->steps_per_tick = config->control_steps_per_tick ? config->control_steps_per_tick : 1u;
        if (server->steps_per_tick > 64) throw std::invalid_argument("control_steps_per_tick must be at most 64");
        server->add_pool(MR_RUN_SOURCE_SYNTHETIC_CHAIN7);
        server->add_pool(MR_RUN_SOURCE_SYNTHETIC_TREE29);
        server->add_pool(MR_RUN_SOURCE_SYNTHETIC_PILE);
        if (server->budget_used > config->hbm_budget_bytes) throw std::invalid_argument("HBM budget exhausted by the slot pools");
    });
    if (rc != 0) return nullptr;
    return server.release();
}

MR_API void mr_server_destroy(MRServerHandle* server) {
    if (server) {
        for (auto& kv : server->pools) cudaStreamSynchronize(kv.second->stream);
        delete server;
    }
}

MR_API int mr_server_capacity(const MRServerHandle* server, uint32_t source, uint32_t* slots, uint32_t* action_count) {
    return guarded([&] {
        if (!server) throw std::invalid_argument("server is null");
        auto it = server->pools.find(source);
        if (it == server->pools.end()) throw std::invalid_argument("unsupported source " + std::to_string(source));
        if (slots) *slots = it->second->capacity;
        if (action_count) *action_count = it->second->na;
    });
}

MR_API int mr_server_submit(MRServerHandle* server, const MRServerRequestC* request, uint64_t* request_id) {
    return guarded([&] {
        if (!server || !request || !request_id) throw std::invalid_argument("null argument");
        Pool& p = server->pool(request->source);
        if (request->env_count == 0 || request->env_count > p.capacity)
            throw std::invalid_argument("env_count must be in [1, " + std::to_string(p.capacity) + "]");
        if (request->horizon == 0) throw std::invalid_argument("horizon must be positive");
        const std::size_t count = static_cast<std::size_t>(request->horizon) * request->env_count * p.na;
        if (count && request->actions == nullptr) throw std::invalid_argument("actions are null");
        auto r = std::make_unique<Request>();
        r->id = server->next_id++;
        r->source = request->source;
        r->envs = request->env_count;
        r->horizon = request->horizon;
        r->seed = request->seed;
        r->host_actions.assign(request->actions, request->actions + count);  // caller span copied
        r->t_submit = now_seconds();
        *request_id = r->id;
        server->pending.push_back(std::move(r));
    });
}

MR_API int mr_server_tick(MRServerHandle* server, uint32_t* active_requests, uint32_t* active_envs) {
    return guarded([&] {
        if (!server) throw std::invalid_argument("server is null");
        // Admission: first come, first served, with backfill of smaller requests.
        for (auto it = server->pending.begin(); it != server->pending.end();) {
            if (server->try_admit(**it)) {
                server->running.push_back(std::move(*it));
                it = server->pending.erase(it);
            } else {
                ++it;
            }
        }
        std::uint32_t reqs = 0, envs = 0;
        for (auto& kv : server->pools) {
            server->scatter_admissions(*kv.second);
            server->launch(*kv.second);
            reqs += static_cast<std::uint32_t>(kv.second->active.size());
            envs += kv.second->tick_env_steps;
        }
        // The tick's one synchronisation: statuses and results are in
        // pinned host memory once the pools' streams drain.
        for (auto& kv : server->pools) check(cudaStreamSynchronize(kv.second->stream), "tick");
        const double t = now_seconds();
        for (auto& kv : server->pools) server->retire(*kv.second, t);
        if (active_requests) *active_requests = reqs;
        if (active_envs) *active_envs = envs;
    });
}

MR_API int mr_server_poll(MRServerHandle* server, MRServerCompletionC* out, uint32_t capacity, uint32_t* count) {
    return guarded([&] {
        if (!server || !count) throw std::invalid_argument("null argument");
        std::uint32_t n = 0;
        while (n < capacity && !server->unreported.empty()) {
            const std::uint64_t id = server->unreported.front();
            server->unreported.erase(server->unreported.begin());
            const Request& r = *server->completed.at(id);
            MRServerCompletionC c{};
            c.request_id = r.id;
            c.source = r.source;
            c.env_count = r.envs;
            c.horizon = r.horizon;
            c.failed_env_steps = r.failed_env_steps;
            c.first_failure_status = r.first_failure_status;
            c.queue_seconds = r.t_admit - r.t_submit;
            c.latency_seconds = r.t_finish - r.t_submit;
            if (out) out[n] = c;
            ++n;
        }
        *count = n;
    });
}

MR_API int mr_server_copy_result(const MRServerHandle* server, uint64_t request_id, float* q, size_t q_count, float* v,
                                 size_t v_count) {
    return guarded([&] {
        if (!server) throw std::invalid_argument("server is null");
        auto it = server->completed.find(request_id);
        if (it == server->completed.end()) throw std::invalid_argument("request " + std::to_string(request_id) + " is not complete");
        const Request& r = *it->second;
        if (q) {
            if (q_count < r.final_q.size()) throw std::invalid_argument("q buffer too small");
            std::memcpy(q, r.final_q.data(), r.final_q.size() * sizeof(float));
        }
        if (v) {
            if (v_count < r.final_v.size()) throw std::invalid_argument("v buffer too small");
            std::memcpy(v, r.final_v.data(), r.final_v.size() * sizeof(float));
        }
    });
}

MR_API int mr_server_release(MRServerHandle* server, uint64_t request_id) {
    return guarded([&] {
        if (!server) throw std::invalid_argument("server is null");
        if (server->completed.erase(request_id) == 0)
            throw std::invalid_argument("request " + std::to_string(request_id) + " is not complete");
    });
}

MR_API int mr_server_stats(const MRServerHandle* server, MRServerStatsC* stats) {
    return guarded([&] {
        if (!server || !stats) throw std::invalid_argument("null argument");
        MRServerStatsC s{};
        s.pending_requests = static_cast<std::uint32_t>(server->pending.size());
        s.running_requests = static_cast<std::uint32_t>(server->running.size());
        s.completed_env_steps = server->completed_env_steps;
        s.hbm_bytes_in_use = server->budget_used;
        for (const auto& kv : server->pools) s.free_slots += static_cast<std::uint32_t>(kv.second->free_slots.size());
        *stats = s;
    });
}

}  // extern "C"
