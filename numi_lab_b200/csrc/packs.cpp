// PolicyPack, PolicyRolloutPack and TaskPack reading and writing (packs.h)
// and the C-ABI entry points that need no rollout: mr_write_policy_pack,
// mr_learning_pack_content_hash, mr_policy_pack_inspect,
// mr_write_policy_rollout_pack, mr_policy_rollout_pack_inspect,
// mr_task_pack_inspect and mr_task_pack_rewrite.
// mr_task_rollout_load_policy_pack (rollout.cu) reads through
// read_policy_pack and installs like mr_task_rollout_set_policy;
// mr_task_rollout_write_policy_rollout_pack (rollout.cu) writes through
// write_policy_rollout_pack.
#include "packs.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <stdexcept>

#include <fcntl.h>
#include <unistd.h>

namespace numi {
namespace rt {
void set_last_error(const std::string& message);
}  // namespace rt

namespace {

constexpr char kMagic[8] = {'M', 'R', 'L', 'E', 'A', 'R', 'N', '\0'};
constexpr std::size_t kHeaderBytes = 32;
constexpr std::uint64_t kMaxPayload = 0xffffffffull;

// Appends little-endian fields (the host is little-endian: x86-64, aarch64).
struct Sink {
    std::vector<std::uint8_t> bytes;
    void raw(const void* p, std::size_t n) {
        const auto* b = static_cast<const std::uint8_t*>(p);
        bytes.insert(bytes.end(), b, b + n);
    }
    void u32(std::uint32_t v) { raw(&v, 4); }
    void u64(std::uint64_t v) { raw(&v, 8); }
    void f32(float v) { raw(&v, 4); }
    void text(const std::string& s) {
        u64(s.size());
        raw(s.data(), s.size());
    }
    void floats(const std::vector<float>& v) {
        u64(v.size());
        if (!v.empty()) raw(v.data(), v.size() * sizeof(float));
    }
    void layers(const std::vector<PolicyPackLayer>& ls) {
        u64(ls.size());
        for (const PolicyPackLayer& l : ls) {
            u32(l.input_count);
            u32(l.output_count);
            u32(l.activation);
            floats(l.weights);
            floats(l.bias);
        }
    }
};

// Bounded reads; every accessor returns false past the end.
struct Source {
    const std::uint8_t* p;
    std::size_t n, at = 0;
    bool raw(void* out, std::size_t k) {
        if (k > n - at) return false;
        std::memcpy(out, p + at, k);
        at += k;
        return true;
    }
    bool u32(std::uint32_t& v) { return raw(&v, 4); }
    bool u64(std::uint64_t& v) { return raw(&v, 8); }
    bool f32(float& v) { return raw(&v, 4); }
    bool text(std::string& s) {
        std::uint64_t k = 0;
        if (!u64(k) || k > n - at || k > kMaxPayload) return false;
        s.assign(reinterpret_cast<const char*>(p + at), static_cast<std::size_t>(k));
        at += static_cast<std::size_t>(k);
        return true;
    }
    bool floats(std::vector<float>& v) {
        std::uint64_t k = 0;
        if (!u64(k) || k > kMaxPayload || k > (n - at) / sizeof(float)) return false;
        v.resize(static_cast<std::size_t>(k));
        return k == 0 || raw(v.data(), v.size() * sizeof(float));
    }
    bool layers(std::vector<PolicyPackLayer>& ls) {
        std::uint64_t k = 0;
        // Each layer takes at least 28 bytes: a corrupt count fails here.
        if (!u64(k) || k > kMaxPayload || k > (n - at) / 28) return false;
        ls.resize(static_cast<std::size_t>(k));
        for (PolicyPackLayer& l : ls)
            if (!u32(l.input_count) || !u32(l.output_count) || !u32(l.activation) || !floats(l.weights) || !floats(l.bias))
                return false;
        return true;
    }
    bool done() const { return at == n; }
};

std::vector<std::uint8_t> encode(const PolicyPackData& d) {
    Sink s;
    s.text(d.id);
    s.u64(d.revision);
    s.floats(d.observation_mean);
    s.floats(d.observation_inverse_std);
    s.layers(d.layers);
    s.floats(d.critic_observation_mean);
    s.floats(d.critic_observation_inverse_std);
    s.layers(d.critic_layers);
    s.floats(d.action_log_std);
    s.floats(d.action_bias);
    s.floats(d.action_scale);
    s.f32(d.observation_clip);
    s.f32(d.action_clip);
    s.u64(d.contract_version);
    s.u64(d.world_fingerprint);
    s.u64(d.task_fingerprint);
    s.u64(d.observation_fingerprint);
    s.u64(d.action_fingerprint);
    return s.bytes;
}

bool contract_exact(const PolicyPackData& d) {
    return d.contract_version == 1 && d.world_fingerprint != 0 && d.task_fingerprint != 0 && d.observation_fingerprint != 0 &&
           d.action_fingerprint != 0;
}

bool decode(const std::uint8_t* bytes, std::size_t count, std::uint32_t version, PolicyPackData& d) {
    Source s{bytes, count};
    if (!(s.text(d.id) && s.u64(d.revision) && s.floats(d.observation_mean) && s.floats(d.observation_inverse_std) &&
          s.layers(d.layers) && s.floats(d.critic_observation_mean) && s.floats(d.critic_observation_inverse_std) &&
          s.layers(d.critic_layers) && s.floats(d.action_log_std) && s.floats(d.action_bias) && s.floats(d.action_scale) &&
          s.f32(d.observation_clip) && s.f32(d.action_clip)))
        return false;
    if (version < 4) return s.done();  // no contract before version 4
    return s.u64(d.contract_version) && s.u64(d.world_fingerprint) && s.u64(d.task_fingerprint) &&
           s.u64(d.observation_fingerprint) && s.u64(d.action_fingerprint) && contract_exact(d) && s.done();
}

bool finite(const std::vector<float>& v) {
    for (float x : v)
        if (!std::isfinite(x)) return false;
    return true;
}

void copy_floats(std::vector<float>& out, const float* p, size_t n, const char* what) {
    if (n != 0 && !p) throw std::invalid_argument(std::string(what) + " is null with a non-zero count");
    out.assign(p, p + n);
}

void copy_layers(std::vector<PolicyPackLayer>& out, const MRPolicyDenseLayerC* ls, size_t n, const char* what) {
    if (n != 0 && !ls) throw std::invalid_argument(std::string(what) + " are null with a non-zero count");
    out.resize(n);
    for (size_t i = 0; i < n; ++i) {
        out[i].input_count = ls[i].input_count;
        out[i].output_count = ls[i].output_count;
        out[i].activation = ls[i].activation;
        copy_floats(out[i].weights, ls[i].weights, ls[i].weight_count, "layer weights");
        copy_floats(out[i].bias, ls[i].bias, ls[i].bias_count, "layer bias");
    }
}

}  // namespace

std::uint64_t learning_pack_hash(const void* bytes, std::size_t count) {
    std::uint64_t h = 14695981039346656037ull;  // FNV-1a 64 offset basis
    const auto* b = static_cast<const std::uint8_t*>(bytes);
    for (std::size_t i = 0; i < count; ++i) {
        h ^= b[i];
        h *= 1099511628211ull;  // FNV 64 prime
    }
    return h == 0 ? 1 : h;
}

PolicyPackData policy_pack_from_c(const MRPolicyPackC& c) {
    PolicyPackData d;
    d.id = c.id ? c.id : "";
    d.revision = c.revision;
    d.contract_version = c.contract_version;
    d.world_fingerprint = c.world_fingerprint;
    d.task_fingerprint = c.task_fingerprint;
    d.observation_fingerprint = c.observation_fingerprint;
    d.action_fingerprint = c.action_fingerprint;
    copy_floats(d.observation_mean, c.observation_mean, c.observation_mean_count, "observation_mean");
    copy_floats(d.observation_inverse_std, c.observation_inverse_standard_deviation,
                c.observation_inverse_standard_deviation_count, "observation_inverse_standard_deviation");
    copy_layers(d.layers, c.layers, c.layer_count, "layers");
    copy_floats(d.critic_observation_mean, c.critic_observation_mean, c.critic_observation_mean_count, "critic_observation_mean");
    copy_floats(d.critic_observation_inverse_std, c.critic_observation_inverse_standard_deviation,
                c.critic_observation_inverse_standard_deviation_count, "critic_observation_inverse_standard_deviation");
    copy_layers(d.critic_layers, c.critic_layers, c.critic_layer_count, "critic_layers");
    copy_floats(d.action_log_std, c.action_log_standard_deviation, c.action_log_standard_deviation_count,
                "action_log_standard_deviation");
    copy_floats(d.action_bias, c.action_bias, c.action_bias_count, "action_bias");
    copy_floats(d.action_scale, c.action_scale, c.action_scale_count, "action_scale");
    d.observation_clip = c.observation_clip;
    d.action_clip = c.action_clip;
    return d;
}

MRPolicyPackC policy_pack_view(const PolicyPackData& d, std::vector<MRPolicyDenseLayerC>& storage) {
    storage.clear();
    storage.reserve(d.layers.size() + d.critic_layers.size());
    auto add = [&](const PolicyPackLayer& l) {
        storage.push_back(MRPolicyDenseLayerC{l.input_count, l.output_count, l.activation, l.weights.data(), l.weights.size(),
                                              l.bias.data(), l.bias.size()});
    };
    for (const PolicyPackLayer& l : d.layers) add(l);
    for (const PolicyPackLayer& l : d.critic_layers) add(l);
    MRPolicyPackC c{};
    c.id = d.id.c_str();
    c.revision = d.revision;
    c.contract_version = d.contract_version;
    c.world_fingerprint = d.world_fingerprint;
    c.task_fingerprint = d.task_fingerprint;
    c.observation_fingerprint = d.observation_fingerprint;
    c.action_fingerprint = d.action_fingerprint;
    c.observation_mean = d.observation_mean.data();
    c.observation_mean_count = d.observation_mean.size();
    c.observation_inverse_standard_deviation = d.observation_inverse_std.data();
    c.observation_inverse_standard_deviation_count = d.observation_inverse_std.size();
    c.layers = storage.data();
    c.layer_count = d.layers.size();
    c.critic_observation_mean = d.critic_observation_mean.data();
    c.critic_observation_mean_count = d.critic_observation_mean.size();
    c.critic_observation_inverse_standard_deviation = d.critic_observation_inverse_std.data();
    c.critic_observation_inverse_standard_deviation_count = d.critic_observation_inverse_std.size();
    c.critic_layers = storage.data() + d.layers.size();
    c.critic_layer_count = d.critic_layers.size();
    c.action_log_standard_deviation = d.action_log_std.data();
    c.action_log_standard_deviation_count = d.action_log_std.size();
    c.action_bias = d.action_bias.data();
    c.action_bias_count = d.action_bias.size();
    c.action_scale = d.action_scale.data();
    c.action_scale_count = d.action_scale.size();
    c.observation_clip = d.observation_clip;
    c.action_clip = d.action_clip;
    return c;
}

void validate_policy_pack(const PolicyPackData& d) {
    if (d.id.empty() || d.revision == 0 || d.layers.empty())
        throw std::invalid_argument("PolicyPack needs an id, a non-zero revision and at least one actor layer");
    if (!contract_exact(d))
        throw std::invalid_argument("PolicyPack semantic contract is not exact (version 1 and non-zero world, task, "
                                    "observation and action fingerprints)");
    if (!std::isfinite(d.observation_clip) || !(d.observation_clip > 0.0f) || !std::isfinite(d.action_clip) ||
        !(d.action_clip > 0.0f))
        throw std::invalid_argument("PolicyPack clips must be positive and finite");
    auto check = [](const std::vector<PolicyPackLayer>& ls, const char* net) {
        for (size_t i = 0; i < ls.size(); ++i) {
            const PolicyPackLayer& l = ls[i];
            if (l.input_count == 0 || l.output_count == 0 || l.activation > MR_POLICY_ACTIVATION_C_SILU ||
                l.weights.size() != static_cast<size_t>(l.input_count) * l.output_count || l.bias.size() != l.output_count ||
                !finite(l.weights) || !finite(l.bias))
                throw std::invalid_argument(std::string("PolicyPack ") + net + " layer " + std::to_string(i) +
                                            " has an invalid shape, activation or value");
        }
    };
    check(d.layers, "actor");
    check(d.critic_layers, "critic");
    if (!d.action_log_std.empty() && d.critic_layers.empty())
        throw std::invalid_argument("a stochastic PolicyPack (action_log_standard_deviation) needs a critic");
    if (!finite(d.observation_mean) || !finite(d.observation_inverse_std) || !finite(d.critic_observation_mean) ||
        !finite(d.critic_observation_inverse_std) || !finite(d.action_log_std) || !finite(d.action_bias) ||
        !finite(d.action_scale))
        throw std::invalid_argument("PolicyPack normalisation and action tables must be finite");
}

namespace {

// Atomically publishes header + payload: a sibling temporary, flushed, renamed.
void publish_pack(const std::vector<std::uint8_t>& payload, std::uint32_t kind, std::uint32_t version, const std::string& path,
                  const char* what) {
    if (path.empty()) throw std::invalid_argument(std::string(what) + " output path is empty");
    if (payload.size() > kMaxPayload) throw std::invalid_argument(std::string(what) + " payload exceeds 4 GiB");
    std::uint8_t header[kHeaderBytes];
    const std::uint64_t bytes = payload.size(), hash = learning_pack_hash(payload.data(), payload.size());
    std::memcpy(header, kMagic, 8);
    std::memcpy(header + 8, &version, 4);
    std::memcpy(header + 12, &kind, 4);
    std::memcpy(header + 16, &bytes, 8);
    std::memcpy(header + 24, &hash, 8);
    std::string tmpl = path + ".tmp.XXXXXX";
    std::vector<char> name(tmpl.begin(), tmpl.end());
    name.push_back('\0');
    const int fd = ::mkstemp(name.data());
    if (fd < 0) throw std::runtime_error("cannot create a temporary beside " + path + ": " + std::strerror(errno));
    auto put = [&](const std::uint8_t* p, std::size_t n) {
        while (n > 0) {
            const ssize_t w = ::write(fd, p, n);
            if (w < 0) {
                if (errno == EINTR) continue;
                return false;
            }
            p += w;
            n -= static_cast<std::size_t>(w);
        }
        return true;
    };
    const bool ok = put(header, kHeaderBytes) && put(payload.data(), payload.size()) && ::fsync(fd) == 0;
    const int err = errno;
    const bool closed = ::close(fd) == 0;
    if (!ok || !closed || ::rename(name.data(), path.c_str()) != 0) {
        const int e = ok && closed ? errno : err;
        ::unlink(name.data());
        throw std::runtime_error("cannot write " + path + ": " + std::strerror(e));
    }
}

struct LoadedPack {
    std::vector<std::uint8_t> payload;
    std::uint32_t version = 0;
    std::uint64_t hash = 0;
};

// Reads a pack of `kind` and version in [oldest, newest], checking the
// length and the payload hash.
LoadedPack load_pack(const std::string& path, std::uint32_t kind, std::uint32_t oldest, std::uint32_t newest, const char* what) {
    std::ifstream in(path, std::ios::binary | std::ios::ate);
    if (!in) throw std::invalid_argument(std::string("cannot open ") + what + " " + path);
    const std::streamoff size = in.tellg();
    if (size < static_cast<std::streamoff>(kHeaderBytes) || static_cast<std::uint64_t>(size) > kHeaderBytes + kMaxPayload)
        throw std::invalid_argument(std::string(what) + " " + path + " has an invalid length");
    in.seekg(0);
    std::uint8_t header[kHeaderBytes];
    if (!in.read(reinterpret_cast<char*>(header), kHeaderBytes)) throw std::invalid_argument(std::string("cannot read the ") + what + " header");
    LoadedPack out;
    std::uint32_t file_kind = 0;
    std::uint64_t bytes = 0;
    std::memcpy(&out.version, header + 8, 4);
    std::memcpy(&file_kind, header + 12, 4);
    std::memcpy(&bytes, header + 16, 8);
    std::memcpy(&out.hash, header + 24, 8);
    if (std::memcmp(header, kMagic, 8) != 0 || file_kind != kind)
        throw std::invalid_argument(std::string("not a ") + what + " (learning-pack magic or artifact kind differs)");
    if (out.version < oldest || out.version > newest)
        throw std::invalid_argument(std::string(what) + " format version " + std::to_string(out.version) + " is not supported (" +
                                    std::to_string(oldest) + (oldest == newest ? "" : "-" + std::to_string(newest)) + ")");
    if (bytes != static_cast<std::uint64_t>(size) - kHeaderBytes)
        throw std::invalid_argument(std::string(what) + " payload length does not match the file");
    out.payload.resize(static_cast<std::size_t>(bytes));
    if (bytes && !in.read(reinterpret_cast<char*>(out.payload.data()), static_cast<std::streamsize>(bytes)))
        throw std::invalid_argument(std::string("cannot read the ") + what + " payload");
    if (learning_pack_hash(out.payload.data(), out.payload.size()) != out.hash)
        throw std::invalid_argument(std::string(what) + " payload hash does not match its header (corrupt file)");
    return out;
}

std::vector<std::uint8_t> encode_rollout(const PolicyRolloutPackData& d) {
    Sink s;
    s.text(d.id);
    s.u64(d.task_fingerprint);
    s.u64(d.policy_fingerprint);
    s.u64(d.policy_revision);
    s.u32(d.environment_count);
    s.u32(d.control_step_count);
    s.u32(d.actor_observation_count);
    s.u32(d.critic_observation_count);
    s.u32(d.action_count);
    s.u32(d.motion_feature_count);
    for (const std::vector<float>* v : {&d.actor_observations, &d.critic_observations, &d.motion_features, &d.teacher_actions,
                                        &d.latents, &d.log_probabilities, &d.values, &d.bootstrap_values})
        s.floats(*v);
    s.u64(d.outcomes.size());
    for (const PolicyOutcome& o : d.outcomes) {
        s.text(o.id);
        s.text(o.unit);
        s.u32(o.direction);
    }
    s.floats(d.outcome_values);
    s.u64(d.transitions.size());
    if (!d.transitions.empty()) s.raw(d.transitions.data(), d.transitions.size() * sizeof(LearningTransition));
    return s.bytes;
}

bool decode_rollout(const std::uint8_t* bytes, std::size_t count, PolicyRolloutPackData& d) {
    Source s{bytes, count};
    if (!(s.text(d.id) && s.u64(d.task_fingerprint) && s.u64(d.policy_fingerprint) && s.u64(d.policy_revision) &&
          s.u32(d.environment_count) && s.u32(d.control_step_count) && s.u32(d.actor_observation_count) &&
          s.u32(d.critic_observation_count) && s.u32(d.action_count) && s.u32(d.motion_feature_count)))
        return false;
    for (std::vector<float>* v : {&d.actor_observations, &d.critic_observations, &d.motion_features, &d.teacher_actions, &d.latents,
                                  &d.log_probabilities, &d.values, &d.bootstrap_values})
        if (!s.floats(*v)) return false;
    std::uint64_t outcomes = 0;
    // Each outcome takes at least 20 bytes: a corrupt count fails here.
    if (!s.u64(outcomes) || outcomes > (s.n - s.at) / 20) return false;
    d.outcomes.resize(static_cast<std::size_t>(outcomes));
    for (PolicyOutcome& o : d.outcomes)
        if (!s.text(o.id) || !s.text(o.unit) || !s.u32(o.direction)) return false;
    std::uint64_t transitions = 0;
    if (!s.floats(d.outcome_values) || !s.u64(transitions) || transitions > (s.n - s.at) / sizeof(LearningTransition)) return false;
    d.transitions.resize(static_cast<std::size_t>(transitions));
    return (transitions == 0 || s.raw(d.transitions.data(), d.transitions.size() * sizeof(LearningTransition))) && s.done();
}

// TaskPack payload (LearningPacks.cpp:1127-1262).
void put_strings(Sink& s, const std::vector<std::string>& v) {
    s.u64(v.size());
    for (const std::string& x : v) s.text(x);
}
void put_f4(Sink& s, const float* f) { s.raw(f, 16); }
void put_f4_list(Sink& s, const std::vector<float>& v) {  // counted four-float records
    s.u64(v.size() / 4);
    if (!v.empty()) s.raw(v.data(), v.size() * sizeof(float));
}

std::vector<std::uint8_t> encode_task(const TaskPackData& d) {
    Sink s;
    s.text(d.id);
    s.raw(d.capacities, sizeof(d.capacities));
    put_strings(s, d.actions);
    s.u64(d.outcomes.size());
    for (const TaskPackOutcome& o : d.outcomes) {
        s.text(o.id);
        s.text(o.unit);
        s.u32(o.source);
        s.u32(o.direction);
        s.u32(o.reward_operation);
    }
    s.u64(d.contact_groups.size());
    for (const TaskPackContactGroup& g : d.contact_groups) {
        s.text(g.id);
        put_strings(s, g.bodies);
        s.raw(&g.support, 1);
        s.raw(&g.forbidden, 1);
        s.text(g.reference_body);
        put_f4(s, g.local_reference);
        s.f32(g.gait_phase_offset);
        s.f32(g.stance_fraction);
        put_f4(s, g.support_patch_bounds);
        s.u32(g.support_patch_width);
        s.u32(g.support_patch_height);
    }
    s.u64(d.joint_groups.size());
    for (const TaskPackJointGroup& g : d.joint_groups) {
        s.text(g.id);
        put_strings(s, g.joints);
    }
    s.u64(d.rewards.size());
    for (const TaskPackReward& r : d.rewards) {
        s.u32(r.operation);
        s.text(r.source_group);
        s.text(r.target);
        s.f32(r.weight);
        put_f4(s, r.parameters);
    }
    s.u64(d.terminations.size());
    for (const TaskPackTermination& t : d.terminations) {
        s.u32(t.operation);
        s.text(t.source_group);
        s.u32(t.reason);
        s.u32(t.priority);
        s.f32(t.threshold);
        s.f32(t.failure_penalty);
        s.u32(t.minimum_band);
        s.u32(t.maximum_band);
    }
    for (const float* c : d.commands) put_f4(s, c);
    s.f32(d.standing_probability);
    s.f32(d.difficulty_sampling_exponent);
    s.f32(d.command_duration[0]);
    s.f32(d.command_duration[1]);
    for (float x : d.pushes) s.f32(x);
    s.text(d.terrain_body);
    put_f4_list(s, d.terrain_sample_offsets);
    put_f4_list(s, d.terrain_reset_translations);
    s.text(d.threat_protected_group);
    for (float x : d.threat) s.f32(x);
    s.text(d.motion_anchor);
    put_strings(s, d.motion_tracked);
    s.u32(d.maximum_episode_steps);
    s.u32(d.difficulty_band_count);
    s.f32(d.interaction_student_authority);
    s.f32(d.interaction_reset_phase_fraction);
    s.floats(d.initial_action_positions);
    s.raw(&d.interaction_control_reference, 1);
    s.raw(&d.interaction_initialize_from_reference, 1);
    s.raw(&d.interaction_align_reference_yaw, 1);
    s.f32(d.base_height_target);
    s.f32(d.gait_period);
    s.f32(d.clearance_target);
    s.f32(d.success_tracking_threshold);
    s.f32(d.support_force_threshold);
    return s.bytes;
}

bool get_strings(Source& s, std::vector<std::string>& v) {
    std::uint64_t k = 0;
    if (!s.u64(k) || k > (s.n - s.at) / 8) return false;  // each string takes at least its 8-byte count
    v.resize(static_cast<std::size_t>(k));
    for (std::string& x : v)
        if (!s.text(x)) return false;
    return true;
}
bool get_f4(Source& s, float* f) { return s.raw(f, 16); }
bool get_f4_list(Source& s, std::vector<float>& v) {
    std::uint64_t k = 0;
    if (!s.u64(k) || k > (s.n - s.at) / 16) return false;
    v.resize(static_cast<std::size_t>(k) * 4);
    return k == 0 || s.raw(v.data(), v.size() * sizeof(float));
}
template <typename T, typename F>
bool get_records(Source& s, std::vector<T>& v, std::size_t least, F&& f) {
    std::uint64_t k = 0;
    if (!s.u64(k) || k > (s.n - s.at) / least) return false;
    v.resize(static_cast<std::size_t>(k));
    for (T& x : v)
        if (!f(x)) return false;
    return true;
}

bool decode_task(const std::uint8_t* bytes, std::size_t count, TaskPackData& d) {
    Source s{bytes, count};
    if (!s.text(d.id) || !s.raw(d.capacities, sizeof(d.capacities)) || !get_strings(s, d.actions)) return false;
    if (!get_records(s, d.outcomes, 28, [&](TaskPackOutcome& o) {
            return s.text(o.id) && s.text(o.unit) && s.u32(o.source) && s.u32(o.direction) && s.u32(o.reward_operation);
        }))
        return false;
    if (!get_records(s, d.contact_groups, 74, [&](TaskPackContactGroup& g) {
            return s.text(g.id) && get_strings(s, g.bodies) && s.raw(&g.support, 1) && s.raw(&g.forbidden, 1) &&
                   s.text(g.reference_body) && get_f4(s, g.local_reference) && s.f32(g.gait_phase_offset) &&
                   s.f32(g.stance_fraction) && get_f4(s, g.support_patch_bounds) && s.u32(g.support_patch_width) &&
                   s.u32(g.support_patch_height);
        }))
        return false;
    if (!get_records(s, d.joint_groups, 16, [&](TaskPackJointGroup& g) { return s.text(g.id) && get_strings(s, g.joints); }))
        return false;
    if (!get_records(s, d.rewards, 40, [&](TaskPackReward& r) {
            return s.u32(r.operation) && s.text(r.source_group) && s.text(r.target) && s.f32(r.weight) && get_f4(s, r.parameters);
        }))
        return false;
    if (!get_records(s, d.terminations, 36, [&](TaskPackTermination& t) {
            return s.u32(t.operation) && s.text(t.source_group) && s.u32(t.reason) && s.u32(t.priority) && s.f32(t.threshold) &&
                   s.f32(t.failure_penalty) && s.u32(t.minimum_band) && s.u32(t.maximum_band);
        }))
        return false;
    for (float* c : d.commands)
        if (!get_f4(s, c)) return false;
    if (!s.f32(d.standing_probability) || !s.f32(d.difficulty_sampling_exponent) || !s.f32(d.command_duration[0]) ||
        !s.f32(d.command_duration[1]))
        return false;
    for (float& x : d.pushes)
        if (!s.f32(x)) return false;
    if (!s.text(d.terrain_body) || !get_f4_list(s, d.terrain_sample_offsets) || !get_f4_list(s, d.terrain_reset_translations) ||
        !s.text(d.threat_protected_group))
        return false;
    for (float& x : d.threat)
        if (!s.f32(x)) return false;
    return s.text(d.motion_anchor) && get_strings(s, d.motion_tracked) && s.u32(d.maximum_episode_steps) &&
           s.u32(d.difficulty_band_count) && s.f32(d.interaction_student_authority) &&
           s.f32(d.interaction_reset_phase_fraction) && s.floats(d.initial_action_positions) &&
           s.raw(&d.interaction_control_reference, 1) && s.raw(&d.interaction_initialize_from_reference, 1) &&
           s.raw(&d.interaction_align_reference_yaw, 1) && s.f32(d.base_height_target) && s.f32(d.gait_period) &&
           s.f32(d.clearance_target) && s.f32(d.success_tracking_threshold) && s.f32(d.support_force_threshold) && s.done();
}

}  // namespace

void validate_task_pack(const TaskPackData& d) {
    auto need = [](bool ok, const char* what) {
        if (!ok) throw std::invalid_argument(what);
    };
    auto fits = [](const std::string& x) { return x.size() <= kMaxPayload; };
    need(!d.id.empty() && fits(d.id) && !d.actions.empty() && d.maximum_episode_steps != 0 && d.difficulty_band_count != 0,
         "TaskPack identity, dimensions, or episode limits are invalid");
    auto probability = [](float x) { return std::isfinite(x) && x >= 0.0f && x <= 1.0f; };
    need(probability(d.interaction_student_authority) && probability(d.interaction_reset_phase_fraction),
         "TaskPack interaction configuration is invalid");
    const float* t = d.threat;
    need(d.threat_protected_group.empty() || (t[0] > 0.0f && t[1] > 0.0f && t[2] >= 0.0f && t[3] > 0.0f && t[4] > 0.0f &&
                                                t[5] > t[4] && t[6] > t[5] && t[7] > 0.0f && t[8] > 0.0f && t[9] > 0.0f),
         "TaskPack threat program is invalid");
    const float* p = d.pushes;  // [4] radius, [5] speed lower, [6] speed upper, [7] height lower, [8] height upper
    const bool ballistics = p[6] > 0.0f;
    need(std::isfinite(p[4]) && p[4] >= 0.0f && std::isfinite(p[5]) && std::isfinite(p[6]) && std::isfinite(p[7]) &&
             std::isfinite(p[8]) && p[5] >= 0.0f && p[6] >= p[5] && (!ballistics || p[5] > 0.0f) && p[8] >= p[7],
         "TaskPack projectile ballistics are invalid");
    for (const TaskPackContactGroup& g : d.contact_groups) {
        const bool patch = g.support_patch_width != 0u || g.support_patch_height != 0u;
        const float* b = g.support_patch_bounds;
        need(!patch || (g.support && g.support_patch_width != 0u && g.support_patch_height != 0u &&
                        static_cast<std::uint64_t>(g.support_patch_width) * g.support_patch_height <= 64u && std::isfinite(b[0]) &&
                        std::isfinite(b[1]) && std::isfinite(b[2]) && std::isfinite(b[3]) && b[2] > b[0] && b[3] > b[1]),
             "TaskPack support patch is invalid");
    }
}

void write_task_pack(const TaskPackData& d, const std::string& path) {
    if (path.empty()) throw std::invalid_argument("TaskPack output path is empty");
    validate_task_pack(d);
    publish_pack(encode_task(d), kTaskPackKind, kTaskPackVersion, path, "TaskPack");
}

TaskPackData read_task_pack(const std::string& path) {
    LoadedPack f = load_pack(path, kTaskPackKind, kTaskPackVersion, kTaskPackVersion, "TaskPack");
    TaskPackData d;
    if (!decode_task(f.payload.data(), f.payload.size(), d)) throw std::invalid_argument("TaskPack payload is malformed");
    d.content_hash = f.hash;
    return d;
}

void write_policy_pack(const PolicyPackData& d, const std::string& path) {
    if (path.empty()) throw std::invalid_argument("PolicyPack output path is empty");
    validate_policy_pack(d);
    publish_pack(encode(d), kPolicyPackKind, kPolicyPackVersion, path, "PolicyPack");
}

PolicyPackData read_policy_pack(const std::string& path) {
    LoadedPack f = load_pack(path, kPolicyPackKind, kPolicyPackOldestVersion, kPolicyPackVersion, "PolicyPack");
    PolicyPackData d;
    if (!decode(f.payload.data(), f.payload.size(), f.version, d)) throw std::invalid_argument("PolicyPack payload is malformed");
    d.format_version = f.version;
    d.content_hash = f.hash;
    return d;
}

std::uint64_t policy_pack_payload_hash(const PolicyPackData& d) {
    const std::vector<std::uint8_t> payload = encode(d);
    return learning_pack_hash(payload.data(), payload.size());
}

LearningTransition learning_transition(const MRTaskTransitionC& t) {
    LearningTransition l{};
    l.reward = t.reward;
    l.timeout_bootstrap_value = t.timeout_bootstrap_value;
    l.done = t.done;
    l.timeout = t.timeout;
    l.physics_error = t.physics_error;
    l.termination_reason = t.termination_reason;
    l.difficulty_band = t.difficulty_band;
    l.terrain_level = t.terrain_level;
    l.impact_sequence_index = t.impact_sequence_index;
    l.impact_event_flags = t.impact_event_flags;
    l.policy_revision = t.policy_revision;
    return l;
}

PolicyRolloutPackData policy_rollout_pack_from_c(const MRPolicyRolloutPackC& c) {
    if (!c.batch) throw std::invalid_argument("policy rollout batch is null");
    const MRPolicyRolloutBatchC& b = *c.batch;
    PolicyRolloutPackData d;
    d.id = c.id ? c.id : "";
    d.task_fingerprint = c.task_fingerprint;
    d.policy_fingerprint = c.policy_fingerprint;
    d.policy_revision = c.policy_revision;
    d.environment_count = c.environment_count;
    d.control_step_count = b.control_step_count;
    d.actor_observation_count = c.actor_observation_count;
    d.critic_observation_count = c.critic_observation_count;
    d.action_count = c.action_count;
    d.motion_feature_count = c.motion_feature_count;
    copy_floats(d.actor_observations, b.actor_observations, b.actor_observation_count, "rollout actor observations");
    copy_floats(d.critic_observations, b.critic_observations, b.critic_observation_count, "rollout critic observations");
    copy_floats(d.motion_features, b.motion_features, b.motion_feature_count, "rollout motion features");
    copy_floats(d.teacher_actions, b.teacher_actions, b.teacher_action_count, "rollout teacher actions");
    copy_floats(d.latents, b.latents, b.latent_count, "rollout latents");
    copy_floats(d.log_probabilities, b.log_probabilities, b.log_probability_count, "rollout log probabilities");
    copy_floats(d.values, b.values, b.value_count, "rollout values");
    copy_floats(d.bootstrap_values, b.bootstrap_values, b.bootstrap_value_count, "rollout bootstrap values");
    if (b.transition_count != 0 && !b.transitions) throw std::invalid_argument("rollout transition pointer is null");
    d.transitions.reserve(b.transition_count);
    for (size_t i = 0; i < b.transition_count; ++i) d.transitions.push_back(learning_transition(b.transitions[i]));
    return d;
}

void validate_policy_rollout_pack(const PolicyRolloutPackData& d) {
    auto need = [](bool ok, const char* what) {
        if (!ok) throw std::invalid_argument(what);
    };
    need(!d.id.empty() && d.id.size() <= kMaxPayload && d.task_fingerprint != 0 && d.policy_fingerprint != 0 &&
             d.policy_revision != 0 && d.environment_count != 0 && d.control_step_count != 0 && d.actor_observation_count != 0 &&
             d.critic_observation_count != 0 && d.action_count != 0,
         "PolicyRolloutPack identity, fingerprints, or dimensions are invalid");
    const std::uint64_t samples = static_cast<std::uint64_t>(d.environment_count) * d.control_step_count;
    auto elements = [&](std::uint32_t per) { return samples * per; };  // counts are 32-bit: no overflow in 64 bits
    bool outcomes_ok = true;
    for (const PolicyOutcome& o : d.outcomes) outcomes_ok = outcomes_ok && !o.id.empty() && o.direction <= 2u;
    need(d.actor_observations.size() == elements(d.actor_observation_count) &&
             d.critic_observations.size() == elements(d.critic_observation_count) &&
             d.motion_features.size() == elements(d.motion_feature_count) &&
             (d.teacher_actions.empty() || d.teacher_actions.size() == elements(d.action_count)) &&
             d.latents.size() == elements(d.action_count) && d.log_probabilities.size() == samples && d.values.size() == samples &&
             d.bootstrap_values.size() == d.environment_count && d.transitions.size() == samples &&
             d.outcome_values.size() == samples * d.outcomes.size() && outcomes_ok,
         "PolicyRolloutPack tensors do not match its declared dimensions");
    bool ok = finite(d.actor_observations) && finite(d.critic_observations) && finite(d.motion_features) && finite(d.teacher_actions) &&
              finite(d.latents) && finite(d.log_probabilities) && finite(d.values) && finite(d.bootstrap_values) &&
              finite(d.outcome_values);
    for (const LearningTransition& t : d.transitions)
        ok = ok && t.policy_revision == d.policy_revision && std::isfinite(t.reward) && std::isfinite(t.timeout_bootstrap_value) &&
             t.done <= 1u && t.timeout <= 1u && t.physics_error <= 1u;
    need(ok, "PolicyRolloutPack contains non-finite or inconsistent samples");
}

void write_policy_rollout_pack(const PolicyRolloutPackData& d, const std::string& path) {
    if (path.empty()) throw std::invalid_argument("PolicyRolloutPack output path is empty");
    validate_policy_rollout_pack(d);
    publish_pack(encode_rollout(d), kPolicyRolloutPackKind, kPolicyRolloutPackVersion, path, "PolicyRolloutPack");
}

PolicyRolloutPackData read_policy_rollout_pack(const std::string& path) {
    LoadedPack f = load_pack(path, kPolicyRolloutPackKind, kPolicyRolloutPackVersion, kPolicyRolloutPackVersion, "PolicyRolloutPack");
    PolicyRolloutPackData d;
    if (!decode_rollout(f.payload.data(), f.payload.size(), d)) throw std::invalid_argument("PolicyRolloutPack payload is malformed");
    validate_policy_rollout_pack(d);
    d.content_hash = f.hash;
    return d;
}

}  // namespace numi

extern "C" {

MR_API int mr_task_pack_inspect(const char* path, MRTaskPackInfoC* info) {
    try {
        if (!path || !path[0]) throw std::invalid_argument("TaskPack path is empty");
        if (!info) throw std::invalid_argument("info is null");
        const numi::TaskPackData d = numi::read_task_pack(path);
        MRTaskPackInfoC o{};
        o.content_hash = d.content_hash;
        o.action_count = static_cast<uint32_t>(d.actions.size());
        o.outcome_count = static_cast<uint32_t>(d.outcomes.size());
        o.contact_group_count = static_cast<uint32_t>(d.contact_groups.size());
        o.joint_group_count = static_cast<uint32_t>(d.joint_groups.size());
        o.reward_count = static_cast<uint32_t>(d.rewards.size());
        o.termination_count = static_cast<uint32_t>(d.terminations.size());
        o.maximum_episode_steps = d.maximum_episode_steps;
        o.difficulty_band_count = d.difficulty_band_count;
        o.terrain_sample_count = static_cast<uint32_t>(d.terrain_sample_offsets.size() / 4);
        o.motion_tracked_body_count = static_cast<uint32_t>(d.motion_tracked.size());
        o.base_height_target = d.base_height_target;
        o.gait_period_seconds = d.gait_period;
        o.clearance_target = d.clearance_target;
        o.support_force_threshold = d.support_force_threshold;
        std::snprintf(o.id, sizeof(o.id), "%s", d.id.c_str());
        *info = o;
        return 0;
    } catch (const std::exception& e) {
        numi::rt::set_last_error(e.what());
        return -1;
    }
}

MR_API int mr_task_pack_rewrite(const char* input_path, const char* output_path) {
    try {
        if (!input_path || !input_path[0] || !output_path || !output_path[0]) throw std::invalid_argument("TaskPack paths are required");
        numi::write_task_pack(numi::read_task_pack(input_path), output_path);
        return 0;
    } catch (const std::exception& e) {
        numi::rt::set_last_error(e.what());
        return -1;
    }
}

MR_API int mr_write_policy_rollout_pack(const MRPolicyRolloutPackC* pack, const char* output_path) {
    try {
        if (!pack) throw std::invalid_argument("policy rollout pack is null");
        if (!output_path || !output_path[0]) throw std::invalid_argument("PolicyRolloutPack output path is empty");
        numi::write_policy_rollout_pack(numi::policy_rollout_pack_from_c(*pack), output_path);
        return 0;
    } catch (const std::exception& e) {
        numi::rt::set_last_error(e.what());
        return -1;
    }
}

MR_API int mr_policy_rollout_pack_inspect(const char* path, MRPolicyRolloutPackInfoC* info, float* parameters, size_t capacity) {
    try {
        if (!path || !path[0]) throw std::invalid_argument("PolicyRolloutPack path is empty");
        if (!info) throw std::invalid_argument("info is null");
        const numi::PolicyRolloutPackData d = numi::read_policy_rollout_pack(path);
        MRPolicyRolloutPackInfoC o{};
        o.task_fingerprint = d.task_fingerprint;
        o.policy_fingerprint = d.policy_fingerprint;
        o.policy_revision = d.policy_revision;
        o.content_hash = d.content_hash;
        o.environment_count = d.environment_count;
        o.control_step_count = d.control_step_count;
        o.actor_observation_count = d.actor_observation_count;
        o.critic_observation_count = d.critic_observation_count;
        o.action_count = d.action_count;
        o.motion_feature_count = d.motion_feature_count;
        o.outcome_count = static_cast<uint32_t>(d.outcomes.size());
        o.has_teacher_actions = d.teacher_actions.empty() ? 0u : 1u;
        o.transition_count = d.transitions.size();
        for (const numi::LearningTransition& t : d.transitions) {
            o.reward_sum += t.reward;
            o.done_count += t.done;
        }
        std::snprintf(o.id, sizeof(o.id), "%s", d.id.c_str());
        if (parameters) {
            size_t at = 0;
            for (const std::vector<float>* v : {&d.actor_observations, &d.latents, &d.log_probabilities, &d.values, &d.bootstrap_values}) {
                if (v->size() > capacity - at) throw std::invalid_argument("parameters capacity is too small");
                std::memcpy(parameters + at, v->data(), v->size() * sizeof(float));
                at += v->size();
            }
        }
        *info = o;
        return 0;
    } catch (const std::exception& e) {
        numi::rt::set_last_error(e.what());
        return -1;
    }
}

MR_API int mr_write_policy_pack(const MRPolicyPackC* policy, const char* policy_pack_path) {
    try {
        if (!policy || !policy_pack_path || !policy_pack_path[0])
            throw std::invalid_argument("a PolicyPack and an output path are required");
        numi::write_policy_pack(numi::policy_pack_from_c(*policy), policy_pack_path);
        return 0;
    } catch (const std::exception& e) {
        numi::rt::set_last_error(std::string("PolicyPack write failed: ") + e.what());
    }
    return -1;
}

MR_API uint64_t mr_learning_pack_content_hash(const void* payload, size_t byte_count) {
    if (!payload && byte_count != 0) return 0;
    return numi::learning_pack_hash(payload, byte_count);
}

MR_API int mr_policy_pack_inspect(const char* policy_pack_path, MRPolicyPackInfoC* info, float* parameters,
                                  size_t parameter_capacity) {
    try {
        if (!policy_pack_path || !info) throw std::invalid_argument("a path and an info output are required");
        const numi::PolicyPackData d = numi::read_policy_pack(policy_pack_path);
        MRPolicyPackInfoC out{};
        out.format_version = d.format_version;
        out.layer_count = static_cast<uint32_t>(d.layers.size());
        out.critic_layer_count = static_cast<uint32_t>(d.critic_layers.size());
        out.observation_count = d.layers.empty() ? 0u : d.layers.front().input_count;
        out.action_count = d.layers.empty() ? 0u : d.layers.back().output_count;
        out.stochastic = d.action_log_std.empty() ? 0u : 1u;
        out.revision = d.revision;
        out.content_hash = d.content_hash;
        out.contract_version = d.contract_version;
        out.world_fingerprint = d.world_fingerprint;
        out.task_fingerprint = d.task_fingerprint;
        out.observation_fingerprint = d.observation_fingerprint;
        out.action_fingerprint = d.action_fingerprint;
        out.observation_clip = d.observation_clip;
        out.action_clip = d.action_clip;
        std::snprintf(out.id, sizeof(out.id), "%s", d.id.c_str());
        // Every FP32 table in wire order.
        std::vector<const std::vector<float>*> tables{&d.observation_mean, &d.observation_inverse_std};
        for (const numi::PolicyPackLayer& l : d.layers) {
            tables.push_back(&l.weights);
            tables.push_back(&l.bias);
        }
        tables.push_back(&d.critic_observation_mean);
        tables.push_back(&d.critic_observation_inverse_std);
        for (const numi::PolicyPackLayer& l : d.critic_layers) {
            tables.push_back(&l.weights);
            tables.push_back(&l.bias);
        }
        tables.push_back(&d.action_log_std);
        tables.push_back(&d.action_bias);
        tables.push_back(&d.action_scale);
        std::size_t total = 0;
        for (const auto* t : tables) total += t->size();
        out.parameter_count = total;
        if (parameters) {
            if (parameter_capacity < total)
                throw std::invalid_argument("parameters holds " + std::to_string(parameter_capacity) + " floats; the pack has " +
                                            std::to_string(total));
            std::size_t at = 0;
            for (const auto* t : tables) {
                if (!t->empty()) std::memcpy(parameters + at, t->data(), t->size() * sizeof(float));
                at += t->size();
            }
        }
        *info = out;
        return 0;
    } catch (const std::exception& e) {
        numi::rt::set_last_error(e.what());
    }
    return -1;
}

}  // extern "C"
