// schedule.cu -- the per-shape launch schedule table (sweep_b200_schedule_*
// in include/sweep_b200.h): shots per CTA, 3-D z chunks and CUDA-graph chunk
// length, recorded per problem shape by the autotuner and read by every plan.
// The only mutable state the library keeps across calls; guarded by a mutex.
#include <array>
#include <map>
#include <mutex>

#include "common.cuh"

namespace sweep {
namespace {

using Key = std::array<int64_t, 12>;

std::mutex g_mu;
std::map<Key, sweep_b200_schedule> g_table;

Key key_of(const sweep_acoustic_desc* d)
{
    return Key{SWEEP_FAMILY_ACOUSTIC, d->ndim, d->B, d->nz, d->ny, d->nx,
               (int64_t)d->pad[0] | (int64_t)d->pad[1] << 20 | (int64_t)d->pad[2] << 40,
               (int64_t)d->pad[3] | (int64_t)d->pad[4] << 20 | (int64_t)d->pad[5] << 40,
               d->vp_stride != 0, 0, 0, 0};
}

Key key_of(const sweep_elastic_desc* d)
{
    return Key{SWEEP_FAMILY_ELASTIC, 2, d->B, d->nz, 1, d->nx,
               (int64_t)d->pad[0] | (int64_t)d->pad[1] << 20,
               (int64_t)d->pad[2] | (int64_t)d->pad[3] << 20,
               d->model_stride != 0, 0, 0, 0};
}

sweep_b200_schedule builtin()
{
    sweep_b200_schedule s{};
    s.graph_steps = -1;
    return s;
}

sweep_b200_schedule lookup(const Key& k)
{
    std::lock_guard<std::mutex> lock(g_mu);
    const auto it = g_table.find(k);
    return it == g_table.end() ? builtin() : it->second;
}

void store(const Key& k, const sweep_b200_schedule& s)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_table[k] = s;
}

}  // namespace

sweep_b200_schedule recorded_schedule(const sweep_acoustic_desc* d) { return lookup(key_of(d)); }
sweep_b200_schedule recorded_schedule(const sweep_elastic_desc* d) { return lookup(key_of(d)); }

int resolve_graph_steps(int recorded)
{
    if (recorded >= 0) return recorded;
    if (const char* e = getenv("SWEEP_B200_GRAPH_STEPS")) {
        const int v = atoi(e);
        if (v >= 0) return v;
    }
    return kGraphStepsDefault;
}

namespace a2d { void schedule_of(const sweep_acoustic_desc* d, sweep_b200_schedule* out); }
namespace a3d { void schedule_of(const sweep_acoustic_desc* d, sweep_b200_schedule* out); }
namespace el2d { void schedule_of(const sweep_elastic_desc* d, sweep_b200_schedule* out); }

}  // namespace sweep

using namespace sweep;

static void check_schedule(const sweep_b200_schedule* s)
{
    SWEEP_REQUIRE(s != nullptr, "null schedule");
    SWEEP_REQUIRE(s->shots_fwd >= 0 && s->shots_fwd <= 16, "schedule: shots_fwd must be 0..16 (got %d)", s->shots_fwd);
    SWEEP_REQUIRE(s->shots_rev >= 0 && s->shots_rev <= 16, "schedule: shots_rev must be 0..16 (got %d)", s->shots_rev);
    SWEEP_REQUIRE(s->z_chunks >= 0 && s->z_chunks <= 64, "schedule: z_chunks must be 0..64 (got %d)", s->z_chunks);
    SWEEP_REQUIRE(s->graph_steps <= 4096, "schedule: graph_steps must be <= 4096 (got %d)", s->graph_steps);
    SWEEP_REQUIRE(s->tile_y == 0 || s->tile_y == 8 || s->tile_y == 16,
                  "schedule: tile_y must be 0 (built-in), 8 or 16 (got %d)", s->tile_y);
}

extern "C" int sweep_b200_schedule_set(int32_t family, const void* desc, const sweep_b200_schedule* s,
                                       char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(desc != nullptr, "null descriptor");
        check_schedule(s);
        sweep_b200_schedule v = *s;
        if (v.graph_steps < 0) v.graph_steps = -1;
        if (family == SWEEP_FAMILY_ACOUSTIC) {
            const auto* d = static_cast<const sweep_acoustic_desc*>(desc);
            SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
            store(key_of(d), v);
        } else {
            SWEEP_REQUIRE(family == SWEEP_FAMILY_ELASTIC, "unknown equation family %d", family);
            store(key_of(static_cast<const sweep_elastic_desc*>(desc)), v);
        }
    });
}

extern "C" int sweep_b200_schedule_get(int32_t family, const void* desc, sweep_b200_schedule* out,
                                       char* err, int32_t err_cap)
{
    return guarded(err, err_cap, [&] {
        SWEEP_REQUIRE(desc != nullptr && out != nullptr, "null argument");
        if (family == SWEEP_FAMILY_ACOUSTIC) {
            const auto* d = static_cast<const sweep_acoustic_desc*>(desc);
            SWEEP_REQUIRE(d->ndim == 2 || d->ndim == 3, "acoustic: ndim %d is not built", d->ndim);
            if (d->ndim == 2) a2d::schedule_of(d, out);
            else a3d::schedule_of(d, out);
        } else {
            SWEEP_REQUIRE(family == SWEEP_FAMILY_ELASTIC, "unknown equation family %d", family);
            el2d::schedule_of(static_cast<const sweep_elastic_desc*>(desc), out);
        }
    });
}

extern "C" int sweep_b200_schedule_clear(void)
{
    std::lock_guard<std::mutex> lock(g_mu);
    g_table.clear();
    return 0;
}
