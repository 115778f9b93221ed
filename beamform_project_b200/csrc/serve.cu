// serve.cu -- served, continuously batched mode.
//
// Host side of bf_serve_* (include/bf_b200.h).  Per-job device state lives in
// one arena (a single allocation of the HBM budget, first-fit over offsets),
// so admission is an exact byte-accounting decision made on the host.  Jobs
// are grouped into kernel classes (grid: antennas x padded beams x window
// kind; tracker: antennas; plus one quantizer class); each class owns a
// device job table at a fixed address.  One served window is:
//   table copy (host -> device, one stream-ordered copy of every class's
//   header and entries) + one CUDA-graph replay of a persistent launch per
//   non-empty class,
// bracketed by CUDA events that give the per-window device time.  The graph
// is captured again only when the set of non-empty classes changes or a
// class outgrows the table capacity it was captured with.
//
// host_only servers (a testing mode) run the same admission, table and state
// logic with no device work: every step completes as soon as it is issued.
#include "bf_internal.cuh"
#include "grid_tc.cuh"
#include "serve.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

struct bf_server;

namespace bf {
namespace {

constexpr uint64_t kAlign = 256;
constexpr int kEventRing = 256;
constexpr int kMirrors = 4;
constexpr int kBranches = 6;
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double kSpeedOfLight = 299792458.0;

uint64_t align_up(uint64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// First-fit allocator over the offsets of one device slab.
class Arena {
public:
    void reset(uint64_t size) {
        size_ = size;
        used_ = peak_ = 0;
        free_.clear();
        if (size > 0) free_[0] = size;
    }
    bool alloc(uint64_t n, uint64_t* off) {
        n = align_up(n);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            *off = it->first;
            const uint64_t rest = it->second - n, start = it->first + n;
            free_.erase(it);
            if (rest > 0) free_[start] = rest;
            used_ += n;
            peak_ = std::max(peak_, used_);
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t n) {
        n = align_up(n);
        used_ -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    uint64_t used() const { return used_; }
    uint64_t peak() const { return peak_; }

private:
    uint64_t size_ = 0, used_ = 0, peak_ = 0;
    std::map<uint64_t, uint64_t> free_;
};

enum ClassKind { kGridClass = 0, kQuantClass = 1, kTrackerClass = 2 };

struct ClassKey {
    int kind, n_ant, nb_pad, rows_q, short_win;
    bool operator<(const ClassKey& o) const {
        return std::tie(kind, n_ant, nb_pad, rows_q, short_win) <
               std::tie(o.kind, o.n_ant, o.nb_pad, o.rows_q, o.short_win);
    }
    bool operator==(const ClassKey& o) const {
        return kind == o.kind && n_ant == o.n_ant && nb_pad == o.nb_pad && rows_q == o.rows_q &&
               short_win == o.short_win;
    }
};

// The quantizer runs per grid class, right after that class's kernel on the
// same graph branch: its key is the grid class's key with the quantizer kind.
ClassKey quant_class_of(const ClassKey& grid) {
    ClassKey q = grid;
    q.kind = kQuantClass;
    return q;
}

uint64_t entry_bytes(int kind) {
    return kind == kGridClass ? sizeof(TcJob) : kind == kQuantClass ? sizeof(QJob) : sizeof(TrJob);
}

int served_nb_pad(uint32_t b) { return b <= 16 ? 16 : b <= 32 ? 32 : b <= 64 ? 64 : 128; }

// Byte layout of one job's arena block.
struct JobLayout {
    uint64_t split = 0, integrated = 0, codes = 0, params = 0;
    uint64_t pos = 0, freq = 0, dirs = 0, kw = 0, traj = 0;
    uint64_t total = 0;
};

struct Job {
    uint64_t id = 0;
    bf_serve_job spec{};
    std::vector<float> pos, freq, dirs, traj;
    std::vector<double> kw;
    int state = BF_JOB_QUEUED;
    JobLayout lay;
    uint64_t off = 0;
    bool has_block = false;
    uint64_t n_steps = 0, next_step = 0, last_step = 0;
    // server steps at submission and at the first launched window
    uint64_t submit_step = 0, admit_step = UINT64_MAX;
    uint64_t n_windows = 0;     // output windows
    ClassKey cls{};
    uint8_t* base = nullptr;    // arena block
    // restored from a checkpoint: windows already served and their results
    // (the prefixes of result_regions), uploaded at admission
    uint64_t resume_step = 0;
    std::vector<uint8_t> resume_results;
};

}  // namespace
}  // namespace bf

using namespace bf;

struct bf_server {
    bf_serve_config cfg{};
    bool host_only = false;
    cudaStream_t stream = nullptr;
    int sms = 148;
    uint8_t* slab = nullptr;
    Arena arena;
    uint8_t* pool[2] = {nullptr, nullptr};   // A = 32, 64
    float* w_scratch = nullptr;              // canonical weights during admission
    std::map<std::pair<int, int>, CUtensorMap> maps;  // (A, rows_q)

    // job bookkeeping
    uint64_t next_id = 1;
    std::map<uint64_t, Job> jobs;
    std::deque<uint64_t> queue;
    std::vector<uint64_t> live;
    std::vector<uint64_t> running;           // every window launched, not yet complete
    std::deque<uint64_t> completions;        // DONE, not yet taken by bf_serve_take_done

    // tables: device buffer and pinned host mirrors with identical layout
    uint64_t table_capacity_bytes = 0;
    uint8_t* d_tables = nullptr;
    uint8_t* h_mirror[kMirrors] = {};
    cudaEvent_t mirror_ev[kMirrors] = {};
    bool mirror_used[kMirrors] = {};
    std::vector<uint8_t> host_mirror;        // host_only mode

    // graph
    struct Captured {
        ClassKey key;
        uint64_t offset;    // of the header in the table buffer
        uint32_t capacity;  // entries
    };
    std::vector<Captured> captured;
    cudaGraphExec_t exec = nullptr;
    uint64_t captures = 0;
    cudaStream_t side[kBranches] = {};       // graph branches (capture only)
    cudaEvent_t fork_ev = nullptr, join_ev[kBranches] = {};

    // step timing
    cudaEvent_t ev_start[kEventRing] = {}, ev_end[kEventRing] = {};
    uint64_t steps = 0, completed_steps = 0;  // steps [0, completed_steps) are complete and timed
    std::vector<float> step_ms;

    // counters
    uint64_t job_windows = 0, submitted = 0, admitted = 0, done = 0, cancelled = 0, rejected = 0;
    uint64_t kernel_launches = 0;
    double predicted_last_us = 0.0;
    double beam_samples = 0.0;
};

namespace bf {
namespace {

JobLayout layout_of(const bf_serve_config& c, const bf_serve_job& j) {
    JobLayout L;
    uint64_t o = 0;
    auto take = [&](uint64_t n) {
        const uint64_t at = o;
        o += align_up(n);
        return at;
    };
    const uint64_t F = c.shard_channels, ns = j.n_shards, A = j.n_ant, B = j.n_beams;
    const uint64_t W = j.n_spectra / j.integration_spectra;
    L.pos = take(A * 3 * sizeof(float));
    if (j.kind == BF_SERVE_GRID) {
        const bf_dims d{j.n_spectra, F, A, B};
        L.split = take(split_weight_bytes(d, ns, served_nb_pad(j.n_beams)));
        L.integrated = take(ns * W * F * B * sizeof(float));
        if (j.quantize) {
            L.codes = take(ns * W * F * B);
            L.params = take(ns * W * ((F + 15) / 16) * ((B + 15) / 16) * 2 * sizeof(float));
        }
        L.freq = take(ns * F * sizeof(float));
        L.dirs = take(B * 3 * sizeof(float));
    } else {
        L.kw = take(ns * F * sizeof(double));
        L.traj = take(B * 4 * sizeof(float));
        L.integrated = take(W * ns * F * B * sizeof(float));
    }
    L.total = o;
    return L;
}

// (offset in the job's block, bytes) of the results of the first `steps`
// served windows: per shard a prefix of integrated (and of codes and
// parameters) for grid jobs, one prefix of integrated for trackers.
std::vector<std::pair<uint64_t, uint64_t>> result_regions(const bf_serve_config& c, const bf_serve_job& j,
                                                          const JobLayout& L, uint64_t steps) {
    std::vector<std::pair<uint64_t, uint64_t>> r;
    const uint64_t F = c.shard_channels, ns = j.n_shards, B = j.n_beams;
    const uint64_t W = j.n_spectra / j.integration_spectra;
    const uint64_t wd = steps * (c.window_spectra / j.integration_spectra);
    if (wd == 0) return r;
    if (j.kind == BF_SERVE_GRID) {
        const uint64_t pt = ((F + 15) / 16) * ((B + 15) / 16) * 2 * sizeof(float);
        for (uint64_t sh = 0; sh < ns; ++sh) {
            r.emplace_back(L.integrated + sh * W * F * B * sizeof(float), wd * F * B * sizeof(float));
            if (j.quantize) {
                r.emplace_back(L.codes + sh * W * F * B, wd * F * B);
                r.emplace_back(L.params + sh * W * pt, wd * pt);
            }
        }
    } else {
        r.emplace_back(L.integrated, wd * ns * F * B * sizeof(float));
    }
    return r;
}

bf_status validate_job(const bf_serve_config& c, const bf_serve_job* j) {
    if (j == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "job must not be null");
    if (j->kind != BF_SERVE_GRID && j->kind != BF_SERVE_TRACKER) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "job kind must be BF_SERVE_GRID or BF_SERVE_TRACKER");
    }
    if (j->n_ant != 32 && j->n_ant != 64) return set_error(BF_ERR_UNSUPPORTED, "served jobs use 32 or 64 antennas");
    if (j->n_shards == 0 || j->n_shards > c.max_shards) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "n_shards must be between 1 and the server's max_shards");
    }
    if (j->kind == BF_SERVE_GRID && (j->n_beams == 0 || j->n_beams > 128)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "grid jobs take 1 to 128 beams");
    }
    if (j->kind == BF_SERVE_TRACKER && (j->n_beams == 0 || j->n_beams > 64)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "tracker jobs take 1 to 64 sources");
    }
    const uint64_t win = c.window_spectra, S = j->integration_spectra;
    if (j->n_spectra == 0 || j->n_spectra % win != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "n_spectra must be a positive multiple of window_spectra");
    }
    if (S == 0 || win % S != 0) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "integration_spectra must divide window_spectra");
    }
    if (j->n_spectra / S > 0x7fffffffull) return set_error(BF_ERR_OVERFLOW, "too many windows in one job");
    if (j->kind == BF_SERVE_GRID && S > 32 && S % 32 != 0) {
        return set_error(BF_ERR_UNSUPPORTED, "grid jobs need integration_spectra below 32 or a multiple of 32");
    }
    if (j->pool_offset % win != 0 || j->pool_offset >= c.pool_spectra) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         "pool_offset must be a multiple of window_spectra below pool_spectra");
    }
    if (j->positions == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "positions must not be null");
    for (uint32_t a = 0; a < 3 * j->n_ant; ++a) {
        if (!std::isfinite(j->positions[a])) return set_error(BF_ERR_INVALID_ARGUMENT, "positions must be finite");
    }
    if (j->frequencies == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "frequencies must not be null");
    for (uint64_t f = 0; f < static_cast<uint64_t>(j->n_shards) * c.shard_channels; ++f) {
        if (!std::isfinite(j->frequencies[f]) || j->frequencies[f] <= 0.f) {
            return set_error(BF_ERR_INVALID_ARGUMENT, "frequencies must be positive and finite");
        }
    }
    if (j->kind == BF_SERVE_GRID) {
        if (j->directions == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "directions must not be null");
        for (uint32_t b = 0; b < j->n_beams; ++b) {
            const float* d = j->directions + 3 * b;
            const double n2 = static_cast<double>(d[0]) * d[0] + static_cast<double>(d[1]) * d[1] +
                              static_cast<double>(d[2]) * d[2];
            if (!std::isfinite(n2) || std::abs(n2 - 1.0) > 1.0e-3) {
                return set_error(BF_ERR_INVALID_ARGUMENT, "beam directions must be finite unit vectors");
            }
        }
    } else {
        if (j->trajectories == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "trajectories must not be null");
        // every window's direction stays on the unit disk (reference
        // tracker_direction throws otherwise)
        const uint64_t W = j->n_spectra / S;
        for (uint32_t s = 0; s < j->n_beams; ++s) {
            const float* tr = j->trajectories + 4 * s;
            for (int i = 0; i < 4; ++i) {
                if (!std::isfinite(tr[i])) return set_error(BF_ERR_INVALID_ARGUMENT, "trajectories must be finite");
            }
            for (uint64_t w = 0; w < W; ++w) {
                const float tf = static_cast<float>(w * S);
                const volatile float l = tr[0] + tf * tr[2];
                const volatile float m = tr[1] + tf * tr[3];
                const volatile float ll = l * l, mm = m * m;
                const float t2 = ll + mm;
                if (!(t2 <= 1.0f)) {
                    return set_error(BF_ERR_INVALID_ARGUMENT, "a tracker trajectory leaves the unit disk");
                }
            }
        }
    }
    return BF_OK;
}

// Windows job j serves in the coming step: up to windows_per_step, stopping
// at its last window and at the end of the voltage pool (a span never wraps).
uint64_t step_windows(const bf_serve_config& c, const Job& j) {
    const uint64_t k = c.windows_per_step > 1 ? c.windows_per_step : 1;
    const uint64_t win = c.window_spectra;
    const uint64_t t0 = (j.spec.pool_offset + j.next_step * win) % c.pool_spectra;
    return std::max<uint64_t>(1, std::min({k, j.n_steps - j.next_step, (c.pool_spectra - t0) / win}));
}

void fill_tables_entry(bf_server* s, const Job& j, uint8_t* hdr, long long* units, uint64_t step,
                       uint64_t n_wsteps, int kind) {
    const bf_serve_config& c = s->cfg;
    const uint64_t win = c.window_spectra, S = j.spec.integration_spectra;
    const uint64_t t0 = (j.spec.pool_offset + step * win) % c.pool_spectra;
    TableHeader* h = reinterpret_cast<TableHeader*>(hdr);
    uint8_t* entry = hdr + sizeof(TableHeader) + static_cast<uint64_t>(h->n_jobs) * entry_bytes(kind);
    if (kind == kGridClass) {
        TcJob e{};
        e.split = j.base + j.lay.split;
        e.integrated = reinterpret_cast<float*>(j.base + j.lay.integrated);
        e.unit_begin = *units;
        e.t0 = static_cast<int>(t0);
        e.n_beams = static_cast<int>(j.spec.n_beams);
        e.beam_stride = e.n_beams;
        e.n_windows = static_cast<int>(j.n_windows);
        e.w0 = static_cast<int>(step * (win / S));
        const long long n = tc_job_tiling(e, static_cast<int>(win * n_wsteps), static_cast<int>(S),
                                          static_cast<int>(c.shard_channels), static_cast<int>(j.spec.n_shards));
        std::memcpy(entry, &e, sizeof(e));
        *units += n;
    } else if (kind == kQuantClass) {
        QJob e{};
        e.integrated = reinterpret_cast<const float*>(j.base + j.lay.integrated);
        e.codes = reinterpret_cast<int8_t*>(j.base + j.lay.codes);
        e.params = reinterpret_cast<float2*>(j.base + j.lay.params);
        e.unit_begin = *units;
        e.n_freq = static_cast<int>(c.shard_channels);
        e.n_beams = static_cast<int>(j.spec.n_beams);
        e.n_windows = static_cast<int>(j.n_windows);
        e.n_win = static_cast<int>(n_wsteps * (win / S));
        e.w0 = static_cast<int>(step * (win / S));
        e.ftiles = static_cast<int>((c.shard_channels + 15) / 16);
        e.btiles = static_cast<int>((j.spec.n_beams + 15) / 16);
        e.n_shards = static_cast<int>(j.spec.n_shards);
        std::memcpy(entry, &e, sizeof(e));
        *units += static_cast<long long>(e.n_shards) * e.n_win * e.ftiles * e.btiles;
    } else {
        TrJob e{};
        e.pos = reinterpret_cast<const float*>(j.base + j.lay.pos);
        e.kw = reinterpret_cast<const double*>(j.base + j.lay.kw);
        e.traj = reinterpret_cast<const float*>(j.base + j.lay.traj);
        e.integrated = reinterpret_cast<float*>(j.base + j.lay.integrated);
        e.unit_begin = *units;
        e.t0 = static_cast<long long>(t0);
        e.n_freq = static_cast<int>(j.spec.n_shards * c.shard_channels);
        e.n_src = static_cast<int>(j.spec.n_beams);
        e.spectra = static_cast<int>(S);
        e.w0 = static_cast<int>(step * (win / S));
        e.n_win = static_cast<int>(n_wsteps * (win / S));
        e.src_groups = (e.n_src + 7) / 8;
        e.fgroups = (e.n_freq + 7) / 8;
        std::memcpy(entry, &e, sizeof(e));
        *units += static_cast<long long>(e.n_win) * e.fgroups * e.src_groups;
    }
    ++h->n_jobs;
    h->n_units = *units;
}

// Completed steps (in order) have their device time collected.
void poll_steps(bf_server* s, bool wait) {
    if (s->host_only) {
        s->completed_steps = s->steps;
        return;
    }
    while (s->completed_steps < s->steps) {
        const int slot = static_cast<int>(s->completed_steps % kEventRing);
        cudaError_t e = wait ? cudaEventSynchronize(s->ev_end[slot]) : cudaEventQuery(s->ev_end[slot]);
        if (e == cudaErrorNotReady) break;
        float ms = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, s->ev_start[slot], s->ev_end[slot]);
        s->step_ms.push_back(ms);
        ++s->completed_steps;
    }
}

void update_done(bf_server* s) {
    size_t keep = 0;
    for (size_t i = 0; i < s->running.size(); ++i) {
        const uint64_t id = s->running[i];
        auto it = s->jobs.find(id);
        if (it == s->jobs.end() || it->second.state != BF_JOB_RUNNING) continue;
        if (it->second.last_step < s->completed_steps) {
            it->second.state = BF_JOB_DONE;
            ++s->done;
            s->completions.push_back(id);
        } else {
            s->running[keep++] = id;
        }
    }
    s->running.resize(keep);
}

// Device-time model of one served window (microseconds), from single-job
// measurements of every class on a B200 at 1965 MHz: a fixed cost per step
// (table copy, graph launch), one per non-empty class (launch ramp and
// tail), and a cost per unit of work.  Grid units: per tile of 128 rows,
// 0.0115 + 0.0105 * (N * K / (256 * 128)) for windows of at least 32
// spectra (a unit is three tiles plus its weight load: x 3), x 1.8 per tile
// for short windows (their epilogue).  Tracker units: 0.015 + S * (0.00016 +
// 0.00004 * tiles) + 2.1e-5 per (source, antenna) weight.
// Resident CTAs per SM of the short-window tracker (registers allow four).
constexpr int kShortTrackerCtasPerSm = 4;
constexpr double kStepUs = 12.0;
constexpr double kClassUs = 8.0;

double job_cost_us(const bf_serve_config& c, const Job& j) {
    const double win = static_cast<double>(c.window_spectra) * static_cast<double>(step_windows(c, j));
    const double S = static_cast<double>(j.spec.integration_spectra);
    const double ch = static_cast<double>(j.spec.n_shards) * c.shard_channels;
    if (j.spec.kind == BF_SERVE_GRID) {
        const double nk = (2.0 * j.cls.nb_pad) * (2.0 * j.spec.n_ant) / (256.0 * 128.0);
        const double tile = 0.0115 + 0.0105 * nk;
        if (j.cls.short_win) {
            const double tiles = std::ceil(win / (4.0 * j.cls.rows_q));
            return ch * tiles * tile * 1.8;
        }
        return ch * std::ceil(win / 128.0) * tile;
    }
    const double n_src = j.spec.n_beams;
    const double groups = std::ceil(n_src / 8.0);
    const double per_window_units = groups * std::ceil(ch / 8.0);
    const double tiles = std::ceil(std::min(8.0, n_src) / 2.0);
    const double unit = 0.015 + S * (0.00016 + 0.00004 * tiles) + 2.1e-5 * std::min(8.0, n_src) * j.spec.n_ant;
    return (win / S) * per_window_units * unit;
}

bf_status encode_pool_map(bf_server* s, int A, int rows_q, CUtensorMap** out) {
    auto key = std::make_pair(A, rows_q);
    auto it = s->maps.find(key);
    if (it == s->maps.end()) {
        CUtensorMap m{};
        if (!s->host_only) {
            const uint64_t F = s->cfg.shard_channels, pool_ch = F * s->cfg.max_shards;
            bf_status st = encode_voltage_map(&m, s->pool[A == 64 ? 1 : 0], A, F, s->cfg.pool_spectra,
                                              s->cfg.max_shards, pool_ch * A, F * A, rows_q);
            if (st != BF_OK) return st;
        }
        it = s->maps.emplace(key, m).first;
    }
    *out = &it->second;
    return BF_OK;
}

// Admits the queue head while it fits; device uploads and weight preparation
// are stream-ordered before the step that first uses them.
double predicted_us(const bf_server* s, const std::vector<uint64_t>& ids, const Job* extra) {
    std::vector<ClassKey> classes;
    double us = kStepUs;
    auto add = [&](const Job& j) {
        us += job_cost_us(s->cfg, j);
        if (std::find(classes.begin(), classes.end(), j.cls) == classes.end()) {
            classes.push_back(j.cls);
            us += kClassUs;
        }
        const ClassKey qk = quant_class_of(j.cls);
        if (j.spec.kind == BF_SERVE_GRID && j.spec.quantize &&
            std::find(classes.begin(), classes.end(), qk) == classes.end()) {
            classes.push_back(qk);
            us += kClassUs;
        }
    };
    for (uint64_t id : ids) add(s->jobs.at(id));
    if (extra != nullptr) add(*extra);
    return us;
}

bf_status admit(bf_server* s) {
    while (!s->queue.empty() && s->live.size() < s->cfg.max_jobs) {
        Job& j = s->jobs.at(s->queue.front());
        if (s->cfg.window_budget_us > 0.f && !s->live.empty() &&
            predicted_us(s, s->live, &j) > s->cfg.window_budget_us) {
            break;
        }
        uint64_t off = 0;
        if (!s->arena.alloc(j.lay.total, &off)) break;
        s->queue.pop_front();
        j.off = off;
        j.has_block = true;
        j.admit_step = s->steps;  // admission runs just before this step's launch
        j.base = reinterpret_cast<uint8_t*>(reinterpret_cast<uintptr_t>(s->slab) + off);
        j.state = BF_JOB_LIVE;
        j.next_step = j.resume_step;
        ++s->admitted;
        s->live.push_back(j.id);
        if (j.resume_step == j.n_steps) {
            // a restored job with every window served: its results are
            // uploaded now and it is done
            s->live.pop_back();
            j.state = BF_JOB_DONE;
            ++s->done;
            s->completions.push_back(j.id);
        }
        if (s->host_only) continue;
        const cudaStream_t st = s->stream;
        const uint64_t A = j.spec.n_ant, F = s->cfg.shard_channels, ns = j.spec.n_shards, B = j.spec.n_beams;
        auto up = [&](uint64_t at, const void* src, uint64_t n) {
            return cuda_status(cudaMemcpyAsync(j.base + at, src, n, cudaMemcpyHostToDevice, st), "job upload");
        };
        BF_RETURN_IF(up(j.lay.pos, j.pos.data(), j.pos.size() * sizeof(float)));
        if (j.spec.kind == BF_SERVE_GRID) {
            BF_RETURN_IF(up(j.lay.freq, j.freq.data(), j.freq.size() * sizeof(float)));
            BF_RETURN_IF(up(j.lay.dirs, j.dirs.data(), j.dirs.size() * sizeof(float)));
            BF_RETURN_IF(launch_generate_weights(st, reinterpret_cast<float*>(j.base + j.lay.pos),
                                                 reinterpret_cast<float*>(j.base + j.lay.freq),
                                                 reinterpret_cast<float*>(j.base + j.lay.dirs), s->w_scratch, ns, F, B,
                                                 A));
            const bf_dims d{j.spec.n_spectra, F, A, B};
            BF_RETURN_IF(launch_prepare_split(st, s->w_scratch, j.base + j.lay.split, d, ns,
                                              served_nb_pad(j.spec.n_beams)));
        } else {
            BF_RETURN_IF(up(j.lay.kw, j.kw.data(), j.kw.size() * sizeof(double)));
            BF_RETURN_IF(up(j.lay.traj, j.traj.data(), j.traj.size() * sizeof(float)));
        }
        if (j.resume_step > 0) {
            uint64_t at = 0;
            for (const auto& reg : result_regions(s->cfg, j.spec, j.lay, j.resume_step)) {
                BF_RETURN_IF(up(reg.first, j.resume_results.data() + at, reg.second));
                at += reg.second;
            }
            if (j.state == BF_JOB_DONE) {
                BF_RETURN_IF(cuda_status(cudaStreamSynchronize(st), "restored results upload"));
            }
        }
    }
    return BF_OK;
}

bf_status capture_graph(bf_server* s, const std::vector<std::pair<ClassKey, uint32_t>>& classes) {
    // table layout for this capture: per class a header and `capacity` entries
    std::vector<bf_server::Captured> cap;
    uint64_t off = 0;
    for (const auto& kc : classes) {
        const uint32_t need = std::max<uint32_t>(16, kc.second);
        uint32_t capacity = 16;
        while (capacity < need) capacity *= 2;
        cap.push_back({kc.first, off, capacity});
        off += align_up(sizeof(TableHeader) + capacity * entry_bytes(kc.first.kind));
    }
    if (off > s->table_capacity_bytes) {
        return set_error(BF_ERR_OVERFLOW, "served job tables exceed the table buffer");
    }
    s->captured = cap;
    ++s->captures;
    if (s->host_only) return BF_OK;
    if (s->exec != nullptr) {
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
    }
    // attributes first: nothing but stream work may run while capturing
    for (const auto& c : cap) {
        if (c.key.kind == kGridClass) {
            CUtensorMap* m = nullptr;
            BF_RETURN_IF(encode_pool_map(s, c.key.n_ant, c.key.rows_q, &m));
            BF_RETURN_IF(launch_grid_tensor_served(s->stream, *m, c.key.n_ant, c.key.nb_pad, nullptr, 0));
        }
    }
    // Classes run on parallel branches of the graph (a fork from the server's
    // stream onto side streams, joined back at the end), so one class's CTAs
    // fill the SMs another class's tail leaves idle; a grid class's quantizer
    // follows it on its branch.
    // Classes never share an SM (each grid CTA holds a whole register file,
    // a tracker CTA half of one), so TMEM allocation never waits.
    cudaGraph_t graph = nullptr;
    BF_RETURN_IF(cuda_status(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal), "begin capture"));
    bf_status st = cuda_status(cudaEventRecord(s->fork_ev, s->stream), "fork the window graph");
    int branch = 0;
    bool used[kBranches] = {};
    auto side = [&]() {
        const int b = branch++ % kBranches;
        if (!used[b]) {
            used[b] = true;
            if (st == BF_OK) st = cuda_status(cudaStreamWaitEvent(s->side[b], s->fork_ev, 0), "branch wait");
        }
        return b;
    };
    auto join = [&]() {
        for (int b = 0; b < kBranches && st == BF_OK; ++b) {
            if (!used[b]) continue;
            st = cuda_status(cudaEventRecord(s->join_ev[b], s->side[b]), "branch done");
            if (st == BF_OK) st = cuda_status(cudaStreamWaitEvent(s->stream, s->join_ev[b], 0), "join the branches");
            used[b] = false;
        }
    };
    // grid and tracker classes on branches, each grid class's quantizer after it
    for (const auto& c : cap) {
        if (st != BF_OK) break;
        if (c.key.kind == kQuantClass) continue;
        const TableHeader* t = reinterpret_cast<const TableHeader*>(s->d_tables + c.offset);
        const int b = side();
        if (st != BF_OK) break;
        if (c.key.kind == kGridClass) {
            CUtensorMap* m = nullptr;
            st = encode_pool_map(s, c.key.n_ant, c.key.rows_q, &m);
            if (st == BF_OK) st = launch_grid_tensor_served(s->side[b], *m, c.key.n_ant, c.key.nb_pad, t, s->sms);
            const ClassKey qk = quant_class_of(c.key);
            for (const auto& q : cap) {
                if (st != BF_OK || !(q.key == qk)) continue;
                st = launch_served_quantize(s->side[b], reinterpret_cast<const TableHeader*>(s->d_tables + q.offset),
                                            s->sms * 8);
            }
        } else {
            const int A = c.key.n_ant;
            const bool short_windows = c.key.short_win != 0;
            st = launch_served_tracker(s->side[b], A, short_windows, s->pool[A == 64 ? 1 : 0],
                                       static_cast<uint64_t>(s->cfg.shard_channels) * s->cfg.max_shards, t,
                                       s->sms * (short_windows ? kShortTrackerCtasPerSm : 2));
        }
    }
    join();
    const cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (st != BF_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    BF_RETURN_IF(cuda_status(e, "end capture"));
    const cudaError_t ie = cudaGraphInstantiate(&s->exec, graph, 0);
    cudaGraphDestroy(graph);
    return cuda_status(ie, "instantiate the served window graph");
}

bf_status step(bf_server* s, uint32_t* n_live) {
    poll_steps(s, false);
    update_done(s);
    // jobs whose windows are all launched, or cancelled, leave the live set
    std::vector<uint64_t> keep;
    for (uint64_t id : s->live) {
        const Job& j = s->jobs.at(id);
        if (j.state == BF_JOB_LIVE) keep.push_back(id);
    }
    s->live.swap(keep);
    BF_RETURN_IF(admit(s));
    if (n_live) *n_live = static_cast<uint32_t>(s->live.size());
    if (s->live.empty()) return BF_OK;

    s->predicted_last_us = predicted_us(s, s->live, nullptr);
    // classes of this step (grid classes, then the quantizer, then trackers)
    std::map<ClassKey, std::vector<uint64_t>> by_class;
    for (uint64_t id : s->live) {
        const Job& j = s->jobs.at(id);
        by_class[j.cls].push_back(id);
        if (j.spec.kind == BF_SERVE_GRID && j.spec.quantize) by_class[quant_class_of(j.cls)].push_back(id);
    }
    std::vector<std::pair<ClassKey, uint32_t>> classes;
    for (const auto& kv : by_class) classes.emplace_back(kv.first, static_cast<uint32_t>(kv.second.size()));
    bool recapture = classes.size() != s->captured.size();
    for (size_t i = 0; !recapture && i < classes.size(); ++i) {
        recapture = !(classes[i].first == s->captured[i].key) || classes[i].second > s->captured[i].capacity;
    }
    if (recapture) BF_RETURN_IF(capture_graph(s, classes));

    // tables into a host mirror
    const int m = static_cast<int>(s->steps % kMirrors);
    uint8_t* mirror = s->host_only ? s->host_mirror.data() : s->h_mirror[m];
    if (!s->host_only && s->mirror_used[m]) {
        BF_RETURN_IF(cuda_status(cudaEventSynchronize(s->mirror_ev[m]), "table mirror reuse"));
    }
    uint64_t used = 0;
    for (const auto& c : s->captured) {
        uint8_t* hdr = mirror + c.offset;
        std::memset(hdr, 0, sizeof(TableHeader));
        long long units = 0;
        for (uint64_t id : by_class[c.key]) {
            const Job& j = s->jobs.at(id);
            fill_tables_entry(s, j, hdr, &units, j.next_step, step_windows(s->cfg, j), c.key.kind);
        }
        used = c.offset + sizeof(TableHeader) + by_class[c.key].size() * entry_bytes(c.key.kind);
    }

    const int slot = static_cast<int>(s->steps % kEventRing);
    if (!s->host_only) {
        if (s->steps >= s->completed_steps + kEventRing) poll_steps(s, true);
        const cudaStream_t st = s->stream;
        BF_RETURN_IF(cuda_status(cudaEventRecord(s->ev_start[slot], st), "record step start"));
        BF_RETURN_IF(cuda_status(cudaMemcpyAsync(s->d_tables, mirror, used, cudaMemcpyHostToDevice, st),
                                 "copy job tables"));
        BF_RETURN_IF(cuda_status(cudaEventRecord(s->mirror_ev[m], st), "record table copy"));
        s->mirror_used[m] = true;
        BF_RETURN_IF(cuda_status(cudaGraphLaunch(s->exec, st), "launch the served window graph"));
        s->kernel_launches += s->captured.size();
        BF_RETURN_IF(cuda_status(cudaEventRecord(s->ev_end[slot], st), "record step end"));
    }
    for (uint64_t id : s->live) {
        Job& j = s->jobs.at(id);
        const uint64_t win = s->cfg.window_spectra;
        const uint64_t ch = static_cast<uint64_t>(j.spec.n_shards) * s->cfg.shard_channels;
        const uint64_t nw = step_windows(s->cfg, j);
        s->beam_samples += static_cast<double>(win * nw) * static_cast<double>(ch) * j.spec.n_beams;
        s->job_windows += nw;
        j.next_step += nw;
        if (j.next_step == j.n_steps) {
            j.state = BF_JOB_RUNNING;
            j.last_step = s->steps;
            s->running.push_back(id);
        }
    }
    ++s->steps;
    if (s->host_only) {
        poll_steps(s, false);
        update_done(s);
    }
    return BF_OK;
}

void destroy(bf_server* s) {
    if (s == nullptr) return;
    if (!s->host_only) {
        if (s->stream) cudaStreamSynchronize(s->stream);
        if (s->exec) cudaGraphExecDestroy(s->exec);
        for (int i = 0; i < kEventRing; ++i) {
            if (s->ev_start[i]) cudaEventDestroy(s->ev_start[i]);
            if (s->ev_end[i]) cudaEventDestroy(s->ev_end[i]);
        }
        for (int i = 0; i < kMirrors; ++i) {
            if (s->mirror_ev[i]) cudaEventDestroy(s->mirror_ev[i]);
            if (s->h_mirror[i]) cudaFreeHost(s->h_mirror[i]);
        }
        cudaFree(s->d_tables);
        cudaFree(s->slab);
        cudaFree(s->pool[0]);
        cudaFree(s->pool[1]);
        cudaFree(s->w_scratch);
        for (int b = 0; b < kBranches; ++b) {
            if (s->join_ev[b]) cudaEventDestroy(s->join_ev[b]);
            if (s->side[b]) cudaStreamDestroy(s->side[b]);
        }
        if (s->fork_ev) cudaEventDestroy(s->fork_ev);
        if (s->stream) cudaStreamDestroy(s->stream);
    }
    delete s;
}

bf_status validate_config(const bf_serve_config& c) {
    if (c.window_spectra == 0 || c.window_spectra % 32 != 0 || c.window_spectra > (1u << 20)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "window_spectra must be a positive multiple of 32");
    }
    if (c.pool_spectra == 0 || c.pool_spectra % c.window_spectra != 0 || c.pool_spectra > (1ull << 30)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "pool_spectra must be a positive multiple of window_spectra");
    }
    if (c.shard_channels == 0 || c.max_shards == 0 || c.max_shards > 64 || c.shard_channels > 65536) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "shard_channels and max_shards must be positive");
    }
    if (c.max_jobs == 0 || c.max_jobs > 65536) return set_error(BF_ERR_INVALID_ARGUMENT, "max_jobs must be 1..65536");
    if (c.hbm_budget_bytes == 0) return set_error(BF_ERR_INVALID_ARGUMENT, "hbm_budget_bytes must be positive");
    if (!(c.window_budget_us >= 0.f)) return set_error(BF_ERR_INVALID_ARGUMENT, "window_budget_us must be >= 0");
    if (c.windows_per_step > 256) return set_error(BF_ERR_INVALID_ARGUMENT, "windows_per_step must be at most 256");
    return BF_OK;
}

bf_status create(const bf_serve_config* cfg, bool host_only, bf_server** out) {
    if (out == nullptr || cfg == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "config and server must not be null");
    *out = nullptr;
    const bf_serve_config& c = *cfg;
    BF_RETURN_IF(validate_config(c));
    std::unique_ptr<bf_server, void (*)(bf_server*)> s(new bf_server(), destroy);
    s->cfg = c;
    s->host_only = host_only;
    s->arena.reset(c.hbm_budget_bytes);
    // table buffer: every class at full capacity (grid classes: 2 antenna
    // counts x 4 beam pads x (long windows + up to 8 short-window row counts);
    // 1 quantizer; 2 trackers)
    const uint64_t per_class = align_up(sizeof(TableHeader) + 2ull * c.max_jobs * sizeof(TrJob));
    s->table_capacity_bytes = per_class * (2 * 4 * 9 + 1 + 2);
    if (host_only) {
        s->host_mirror.assign(s->table_capacity_bytes, 0);
        *out = s.release();
        return BF_OK;
    }
    BF_RETURN_IF(cuda_status(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "create stream"));
    for (int b = 0; b < kBranches; ++b) {
        BF_RETURN_IF(cuda_status(cudaStreamCreateWithFlags(&s->side[b], cudaStreamNonBlocking), "create stream"));
        BF_RETURN_IF(cuda_status(cudaEventCreateWithFlags(&s->join_ev[b], cudaEventDisableTiming), "create event"));
    }
    BF_RETURN_IF(cuda_status(cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming), "create event"));
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, dev);
    BF_RETURN_IF(cuda_status(cudaMalloc(&s->slab, c.hbm_budget_bytes), "allocate the job arena"));
    const uint64_t pool_ch = static_cast<uint64_t>(c.shard_channels) * c.max_shards;
    for (int i = 0; i < 2; ++i) {
        const uint64_t A = i == 0 ? 32 : 64;
        BF_RETURN_IF(cuda_status(cudaMalloc(&s->pool[i], c.pool_spectra * pool_ch * A), "allocate a voltage pool"));
        const bf_dims d{c.pool_spectra, pool_ch, A, 1};
        BF_RETURN_IF(launch_generate(s->stream, c.pool_seed + A, 0, c.pool_scale, nullptr, 1, s->pool[i], d));
    }
    BF_RETURN_IF(cuda_status(cudaMalloc(&s->w_scratch, c.max_shards * 128ull * c.shard_channels * 64ull * 8ull),
                             "allocate the weight scratch"));
    BF_RETURN_IF(cuda_status(cudaMalloc(&s->d_tables, s->table_capacity_bytes), "allocate the job tables"));
    for (int i = 0; i < kMirrors; ++i) {
        BF_RETURN_IF(cuda_status(cudaMallocHost(&s->h_mirror[i], s->table_capacity_bytes), "allocate a table mirror"));
        BF_RETURN_IF(cuda_status(cudaEventCreateWithFlags(&s->mirror_ev[i], cudaEventDisableTiming), "create event"));
    }
    for (int i = 0; i < kEventRing; ++i) {
        BF_RETURN_IF(cuda_status(cudaEventCreate(&s->ev_start[i]), "create event"));
        BF_RETURN_IF(cuda_status(cudaEventCreate(&s->ev_end[i]), "create event"));
    }
    BF_RETURN_IF(cuda_status(cudaStreamSynchronize(s->stream), "fill the voltage pools"));
    *out = s.release();
    return BF_OK;
}

}  // namespace
}  // namespace bf

namespace bf {
namespace {

// A validated job (host inputs copied), not yet queued.
bf_status make_job(bf_server* s, const bf_serve_job* job, Job* out) {
    BF_RETURN_IF(validate_job(s->cfg, job));
    Job& j = *out;
    j.spec = *job;
    j.lay = layout_of(s->cfg, *job);
    if (j.lay.total > s->cfg.hbm_budget_bytes) {
        ++s->rejected;
        return set_error(BF_ERR_RESOURCE, "the job's device state exceeds the server's HBM budget");
    }
    const uint64_t F = static_cast<uint64_t>(job->n_shards) * s->cfg.shard_channels;
    j.pos.assign(job->positions, job->positions + 3 * job->n_ant);
    j.freq.assign(job->frequencies, job->frequencies + F);
    if (job->kind == BF_SERVE_GRID) {
        j.dirs.assign(job->directions, job->directions + 3 * job->n_beams);
        j.cls = ClassKey{kGridClass, static_cast<int>(job->n_ant), served_nb_pad(job->n_beams),
                         small_window_rows(static_cast<int>(job->integration_spectra)),
                         job->integration_spectra < 32 ? 1 : 0};
    } else {
        j.traj.assign(job->trajectories, job->trajectories + 4 * job->n_beams);
        j.kw.resize(F);
        for (uint64_t f = 0; f < F; ++f) j.kw[f] = kTwoPi * static_cast<double>(j.freq[f]) / kSpeedOfLight;
        j.cls = ClassKey{kTrackerClass, static_cast<int>(job->n_ant), 0, 0, job->integration_spectra <= 16 ? 1 : 0};
    }
    j.spec.positions = j.spec.frequencies = j.spec.directions = j.spec.trajectories = nullptr;
    j.n_steps = job->n_spectra / s->cfg.window_spectra;
    j.n_windows = job->n_spectra / job->integration_spectra;
    return BF_OK;
}

// ---- job checkpoints ----
// Image (little-endian, no padding): "BFSRVCK1", version, the job's scalar
// fields, the windows served, the server settings its voltages depend on
// (window, shard channels, max shards, pool rows, seed and scale), the job's
// host arrays (positions, frequencies, directions or trajectories), the
// results of the served windows (the prefixes of result_regions, in order),
// and an FNV-1a 64 checksum of everything before it.
constexpr char kImageMagic[8] = {'B', 'F', 'S', 'R', 'V', 'C', 'K', '1'};
constexpr uint32_t kImageVersion = 1;

uint64_t fnv1a(const uint8_t* p, uint64_t n) {
    uint64_t h = 14695981039346656037ull;
    for (uint64_t i = 0; i < n; ++i) h = (h ^ p[i]) * 1099511628211ull;
    return h;
}

struct ImageHead {
    uint32_t kind, n_ant, n_shards, n_beams, quantize;
    uint64_t n_spectra, spectra, pool_offset, steps_done;
    uint32_t window_spectra, shard_channels, max_shards, pool_scale_bits;
    uint64_t pool_spectra, pool_seed;
};

class ImageOut {
public:
    explicit ImageOut(std::vector<uint8_t>* b) : b_(b) {}
    template <typename T>
    void put(const T& v) { raw(&v, sizeof(T)); }
    void raw(const void* p, size_t n) {
        const auto* c = static_cast<const uint8_t*>(p);
        b_->insert(b_->end(), c, c + n);
    }

private:
    std::vector<uint8_t>* b_;
};

class ImageIn {
public:
    ImageIn(const uint8_t* p, uint64_t n) : p_(p), n_(n) {}
    template <typename T>
    bool get(T* v) { return raw(v, sizeof(T)); }
    bool raw(void* dst, uint64_t n) {
        if (n > n_ - at_) return false;
        std::memcpy(dst, p_ + at_, n);
        at_ += n;
        return true;
    }
    uint64_t left() const { return n_ - at_; }

private:
    const uint8_t* p_;
    uint64_t n_, at_ = 0;
};

void put_head(ImageOut& o, const ImageHead& h) {
    o.raw(kImageMagic, sizeof(kImageMagic));
    o.put(kImageVersion);
    o.put(h.kind); o.put(h.n_ant); o.put(h.n_shards); o.put(h.n_beams); o.put(h.quantize);
    o.put(h.n_spectra); o.put(h.spectra); o.put(h.pool_offset); o.put(h.steps_done);
    o.put(h.window_spectra); o.put(h.shard_channels); o.put(h.max_shards); o.put(h.pool_scale_bits);
    o.put(h.pool_spectra); o.put(h.pool_seed);
}

bool get_head(ImageIn& in, ImageHead* h) {
    char magic[8];
    uint32_t version = 0;
    if (!in.raw(magic, sizeof(magic)) || std::memcmp(magic, kImageMagic, sizeof(magic)) != 0) return false;
    if (!in.get(&version) || version != kImageVersion) return false;
    return in.get(&h->kind) && in.get(&h->n_ant) && in.get(&h->n_shards) && in.get(&h->n_beams) &&
           in.get(&h->quantize) && in.get(&h->n_spectra) && in.get(&h->spectra) && in.get(&h->pool_offset) &&
           in.get(&h->steps_done) && in.get(&h->window_spectra) && in.get(&h->shard_channels) &&
           in.get(&h->max_shards) && in.get(&h->pool_scale_bits) && in.get(&h->pool_spectra) &&
           in.get(&h->pool_seed);
}

uint32_t float_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, sizeof(u));
    return u;
}

uint64_t regions_bytes(const std::vector<std::pair<uint64_t, uint64_t>>& r) {
    uint64_t n = 0;
    for (const auto& x : r) n += x.second;
    return n;
}

// windows whose results a checkpoint of j carries
uint64_t served_steps(const Job& j) {
    return j.state == BF_JOB_QUEUED ? j.resume_step : j.next_step;
}

bf_status build_image(bf_server* s, const Job& j, std::vector<uint8_t>* img) {
    const bf_serve_config& c = s->cfg;
    const uint64_t done = served_steps(j);
    ImageHead h{static_cast<uint32_t>(j.spec.kind), j.spec.n_ant, j.spec.n_shards, j.spec.n_beams,
                static_cast<uint32_t>(j.spec.quantize != 0), j.spec.n_spectra, j.spec.integration_spectra,
                j.spec.pool_offset, done, c.window_spectra, c.shard_channels, c.max_shards,
                float_bits(c.pool_scale), c.pool_spectra, c.pool_seed};
    ImageOut o(img);
    put_head(o, h);
    o.raw(j.pos.data(), j.pos.size() * sizeof(float));
    o.raw(j.freq.data(), j.freq.size() * sizeof(float));
    if (j.spec.kind == BF_SERVE_GRID) o.raw(j.dirs.data(), j.dirs.size() * sizeof(float));
    else o.raw(j.traj.data(), j.traj.size() * sizeof(float));
    const auto regions = result_regions(c, j.spec, j.lay, done);
    const uint64_t at = img->size();
    img->resize(at + regions_bytes(regions));
    if (j.state == BF_JOB_QUEUED) {
        if (!j.resume_results.empty()) std::memcpy(img->data() + at, j.resume_results.data(), j.resume_results.size());
    } else if (!s->host_only) {
        uint64_t o2 = at;
        for (const auto& r : regions) {
            BF_RETURN_IF(cuda_status(cudaMemcpy(img->data() + o2, j.base + r.first, r.second, cudaMemcpyDeviceToHost),
                                     "checkpoint results copy"));
            o2 += r.second;
        }
    }
    const uint64_t sum = fnv1a(img->data(), img->size());
    ImageOut(img).put(sum);
    return BF_OK;
}

uint64_t image_bytes(const bf_serve_config& c, const Job& j) {
    const uint64_t arrays = j.pos.size() + j.freq.size() + (j.spec.kind == BF_SERVE_GRID ? j.dirs.size() : j.traj.size());
    const uint64_t head = sizeof(kImageMagic) + sizeof(uint32_t) * 10 + sizeof(uint64_t) * 6;
    return head + arrays * sizeof(float) + regions_bytes(result_regions(c, j.spec, j.lay, served_steps(j))) +
           sizeof(uint64_t);
}

void enqueue(bf_server* s, Job&& j, uint64_t* job_id) {
    j.id = s->next_id++;
    j.submit_step = s->steps;
    if (job_id) *job_id = j.id;
    s->queue.push_back(j.id);
    s->jobs.emplace(j.id, std::move(j));
    ++s->submitted;
}

}  // namespace
}  // namespace bf

extern "C" {

BF_API uint64_t bf_serve_job_bytes(const bf_serve_config* config, const bf_serve_job* job) {
    if (config == nullptr || job == nullptr || validate_config(*config) != BF_OK ||
        validate_job(*config, job) != BF_OK) {
        return 0;
    }
    return layout_of(*config, *job).total;
}

static bf_status bf_serve_create_impl(const bf_serve_config* config, bf_server** server) {
    clear_error();
    return create(config, false, server);
}

BF_API bf_status bf_serve_create(const bf_serve_config* config, bf_server** server) {
    try {
        return bf_serve_create_impl(config, server);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

// Scheduler-only server (no device work), used to test admission and tables
// without a GPU.
static bf_status bf_serve_create_host_only_impl(const bf_serve_config* config, bf_server** server) {
    clear_error();
    return create(config, true, server);
}

BF_API bf_status bf_serve_create_host_only(const bf_serve_config* config, bf_server** server) {
    try {
        return bf_serve_create_host_only_impl(config, server);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

BF_API bf_status bf_serve_destroy(bf_server* server) {
    clear_error();
    destroy(server);
    return BF_OK;
}

static bf_status bf_serve_submit_impl(bf_server* s, const bf_serve_job* job, uint64_t* job_id) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    Job j;
    BF_RETURN_IF(make_job(s, job, &j));
    enqueue(s, std::move(j), job_id);
    return BF_OK;
}

BF_API bf_status bf_serve_submit(bf_server* s, const bf_serve_job* job, uint64_t* job_id) {
    try {
        return bf_serve_submit_impl(s, job, job_id);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_step_impl(bf_server* s, uint32_t* n_live) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    return step(s, n_live);
}

BF_API bf_status bf_serve_step(bf_server* s, uint32_t* n_live) {
    try {
        return bf_serve_step_impl(s, n_live);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_poll_impl(bf_server* s, uint64_t job_id, int32_t* state) {
    clear_error();
    if (s == nullptr || state == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server and state must not be null");
    poll_steps(s, false);
    update_done(s);
    auto it = s->jobs.find(job_id);
    *state = it == s->jobs.end() ? BF_JOB_UNKNOWN : it->second.state;
    return BF_OK;
}

BF_API bf_status bf_serve_poll(bf_server* s, uint64_t job_id, int32_t* state) {
    try {
        return bf_serve_poll_impl(s, job_id, state);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_job_info_impl(bf_server* s, uint64_t job_id, bf_serve_job_info* info) {
    clear_error();
    if (s == nullptr || info == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server and info must not be null");
    poll_steps(s, false);
    update_done(s);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return set_error(BF_ERR_OUT_OF_RANGE, "unknown served job id");
    const Job& j = it->second;
    *info = bf_serve_job_info{};
    info->state = j.state;
    info->submit_step = j.submit_step;
    info->admit_step = j.admit_step;
    const bool all = j.state == BF_JOB_RUNNING || (j.state == BF_JOB_DONE && j.n_steps > j.resume_step);
    info->last_step = all ? j.last_step : UINT64_MAX;
    info->windows_launched = j.next_step - j.resume_step;
    return BF_OK;
}

BF_API bf_status bf_serve_job_info_get(bf_server* s, uint64_t job_id, bf_serve_job_info* info) {
    try {
        return bf_serve_job_info_impl(s, job_id, info);
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_result_impl(bf_server* s, uint64_t job_id, float** integrated, int8_t** codes, float** params,
                                 uint64_t* n_windows) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    poll_steps(s, false);
    update_done(s);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return set_error(BF_ERR_OUT_OF_RANGE, "unknown job id");
    const Job& j = it->second;
    if (j.state != BF_JOB_DONE) return set_error(BF_ERR_LOGIC, "the job's results are not complete");
    if (integrated) *integrated = reinterpret_cast<float*>(j.base + j.lay.integrated);
    if (codes) *codes = j.spec.quantize && j.spec.kind == BF_SERVE_GRID ? reinterpret_cast<int8_t*>(j.base + j.lay.codes) : nullptr;
    if (params) *params = j.spec.quantize && j.spec.kind == BF_SERVE_GRID ? reinterpret_cast<float*>(j.base + j.lay.params) : nullptr;
    if (n_windows) *n_windows = j.n_windows;
    return BF_OK;
}

BF_API bf_status bf_serve_result(bf_server* s, uint64_t job_id, float** integrated, int8_t** codes, float** params,
                                 uint64_t* n_windows) {
    try {
        return bf_serve_result_impl(s, job_id, integrated, codes, params, n_windows);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_cancel_impl(bf_server* s, uint64_t job_id) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return set_error(BF_ERR_OUT_OF_RANGE, "unknown job id");
    Job& j = it->second;
    if (j.state == BF_JOB_QUEUED) {
        s->queue.erase(std::find(s->queue.begin(), s->queue.end(), job_id));
    } else if (j.state == BF_JOB_LIVE) {
        // it leaves the live set at the next step; the GPU may use its state
        // until the last step already issued completes
        j.last_step = s->steps - 1;
    } else {
        return set_error(BF_ERR_LOGIC, "only queued or live jobs can be cancelled");
    }
    j.state = BF_JOB_CANCELLED;
    ++s->cancelled;
    return BF_OK;
}

BF_API bf_status bf_serve_cancel(bf_server* s, uint64_t job_id) {
    try {
        return bf_serve_cancel_impl(s, job_id);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_release_impl(bf_server* s, uint64_t job_id) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    poll_steps(s, false);
    update_done(s);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return set_error(BF_ERR_OUT_OF_RANGE, "unknown job id");
    Job& j = it->second;
    if (j.state != BF_JOB_DONE && j.state != BF_JOB_CANCELLED) {
        return set_error(BF_ERR_LOGIC, "only done or cancelled jobs can be released");
    }
    if (j.has_block) {
        if (j.last_step >= s->completed_steps) poll_steps(s, true);  // a cancelled job still in flight
        s->arena.release(j.off, j.lay.total);
    }
    s->live.erase(std::remove(s->live.begin(), s->live.end(), job_id), s->live.end());
    s->completions.erase(std::remove(s->completions.begin(), s->completions.end(), job_id), s->completions.end());
    s->jobs.erase(it);
    return BF_OK;
}

BF_API bf_status bf_serve_release(bf_server* s, uint64_t job_id) {
    try {
        return bf_serve_release_impl(s, job_id);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_sync_impl(bf_server* s) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    if (!s->host_only) {
        BF_RETURN_IF(cuda_status(cudaStreamSynchronize(s->stream), "served stream"));
        uint32_t code = 0;
        BF_RETURN_IF(take_tc_error(&code));
        if (code != 0) return set_error(BF_ERR_TIMEOUT, "a served kernel's bounded wait ran out (code " +
                                                            std::to_string(code) + ")");
    }
    poll_steps(s, true);
    update_done(s);
    return BF_OK;
}

BF_API bf_status bf_serve_sync(bf_server* s) {
    try {
        return bf_serve_sync_impl(s);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_stats_get_impl(bf_server* s, bf_serve_stats* out) {
    clear_error();
    if (s == nullptr || out == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server and stats must not be null");
    poll_steps(s, true);
    update_done(s);
    bf_serve_stats st{};
    st.steps = s->steps;
    st.steps_timed = s->step_ms.size();
    st.job_windows = s->job_windows;
    st.jobs_submitted = s->submitted;
    st.jobs_admitted = s->admitted;
    st.jobs_done = s->done;
    st.jobs_cancelled = s->cancelled;
    st.jobs_rejected = s->rejected;
    st.live_jobs = s->live.size();
    st.queued_jobs = s->queue.size();
    st.arena_bytes_in_use = s->arena.used();
    st.arena_bytes_peak = s->arena.peak();
    st.graph_captures = s->captures;
    st.beam_samples = s->beam_samples;
    st.kernel_launches = s->kernel_launches;
    st.predicted_ms_last = s->predicted_last_us * 1e-3;
    if (!s->step_ms.empty()) {
        std::vector<float> v = s->step_ms;
        double total = 0.0;
        for (float x : v) total += x;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const size_t i = static_cast<size_t>(std::ceil(p * v.size())) - 1;
            return static_cast<double>(v[std::min(i, v.size() - 1)]);
        };
        st.step_ms_total = total;
        st.step_ms_p50 = pct(0.50);
        st.step_ms_p99 = pct(0.99);
        st.step_ms_max = v.back();
    }
    *out = st;
    return BF_OK;
}

BF_API bf_status bf_serve_stats_get(bf_server* s, bf_serve_stats* out) {
    try {
        return bf_serve_stats_get_impl(s, out);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_step_times_impl(bf_server* s, float* out, uint64_t capacity, uint64_t* count) {
    clear_error();
    if (s == nullptr || count == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server and count must not be null");
    poll_steps(s, true);
    *count = s->step_ms.size();
    if (out != nullptr) std::copy_n(s->step_ms.begin(), std::min<uint64_t>(capacity, s->step_ms.size()), out);
    return BF_OK;
}

BF_API bf_status bf_serve_step_times(bf_server* s, float* out, uint64_t capacity, uint64_t* count) {
    try {
        return bf_serve_step_times_impl(s, out, capacity, count);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

BF_API bf_status bf_serve_take_done(bf_server* s, uint64_t* ids, uint64_t capacity, uint64_t* count) {
    clear_error();
    if (s == nullptr || count == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server and count must not be null");
    poll_steps(s, false);
    update_done(s);
    uint64_t n = 0;
    while (n < capacity && ids != nullptr && !s->completions.empty()) {
        ids[n++] = s->completions.front();
        s->completions.pop_front();
    }
    *count = n;
    return BF_OK;
}

BF_API void* bf_serve_stream(bf_server* s) { return s == nullptr ? nullptr : static_cast<void*>(s->stream); }

BF_API bf_status bf_serve_pool(bf_server* s, uint64_t n_ant, uint8_t** pool, uint64_t* pool_spectra,
                               uint64_t* pool_channels) {
    clear_error();
    if (s == nullptr || pool == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server and pool must not be null");
    if (n_ant != 32 && n_ant != 64) return set_error(BF_ERR_INVALID_ARGUMENT, "served pools hold 32 or 64 antennas");
    if (s->host_only) return set_error(BF_ERR_LOGIC, "a host-only server has no device pools");
    *pool = s->pool[n_ant == 64 ? 1 : 0];
    if (pool_spectra != nullptr) *pool_spectra = s->cfg.pool_spectra;
    if (pool_channels != nullptr) *pool_channels = static_cast<uint64_t>(s->cfg.shard_channels) * s->cfg.max_shards;
    return BF_OK;
}

static bf_status bf_serve_checkpoint_impl(bf_server* s, uint64_t job_id, void* buffer, uint64_t capacity,
                                          uint64_t* bytes) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    poll_steps(s, false);
    update_done(s);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) return set_error(BF_ERR_OUT_OF_RANGE, "unknown job id");
    const Job& j = it->second;
    if (j.state == BF_JOB_CANCELLED) return set_error(BF_ERR_LOGIC, "a cancelled job has no checkpoint");
    const uint64_t n = image_bytes(s->cfg, j);
    if (bytes) *bytes = n;
    if (buffer == nullptr) return BF_OK;
    if (capacity < n) return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint buffer is smaller than the image");
    if (j.state != BF_JOB_QUEUED && !s->host_only) {
        // the windows already launched for this job complete first
        poll_steps(s, true);
        BF_RETURN_IF(cuda_status(cudaStreamSynchronize(s->stream), "checkpoint wait"));
    }
    std::vector<uint8_t> img;
    img.reserve(n);
    BF_RETURN_IF(build_image(s, j, &img));
    if (img.size() != n) return set_error(BF_ERR_LOGIC, "internal error: checkpoint size");
    std::memcpy(buffer, img.data(), n);
    return BF_OK;
}

BF_API bf_status bf_serve_checkpoint(bf_server* s, uint64_t job_id, void* buffer, uint64_t capacity,
                                     uint64_t* bytes) {
    try {
        return bf_serve_checkpoint_impl(s, job_id, buffer, capacity, bytes);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

static bf_status bf_serve_restore_impl(bf_server* s, const void* image, uint64_t bytes, uint64_t* job_id) {
    clear_error();
    if (s == nullptr) return set_error(BF_ERR_INVALID_ARGUMENT, "server must not be null");
    if (image == nullptr || bytes < sizeof(uint64_t)) return set_error(BF_ERR_INVALID_ARGUMENT, "no checkpoint image");
    const auto* p = static_cast<const uint8_t*>(image);
    uint64_t sum = 0;
    std::memcpy(&sum, p + bytes - sizeof(uint64_t), sizeof(uint64_t));
    if (fnv1a(p, bytes - sizeof(uint64_t)) != sum) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint image is damaged (checksum)");
    }
    ImageIn in(p, bytes - sizeof(uint64_t));
    ImageHead h{};
    if (!get_head(in, &h)) return set_error(BF_ERR_INVALID_ARGUMENT, "not a served-job checkpoint image");
    const bf_serve_config& c = s->cfg;
    if (h.window_spectra != c.window_spectra || h.shard_channels != c.shard_channels ||
        h.max_shards != c.max_shards || h.pool_scale_bits != float_bits(c.pool_scale) ||
        h.pool_spectra != c.pool_spectra || h.pool_seed != c.pool_seed) {
        return set_error(BF_ERR_INVALID_ARGUMENT,
                         "the checkpoint comes from a server with other window, shard or pool settings");
    }
    if (h.n_ant > 1024 || h.n_shards > 64 || h.n_beams > 1024) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint job fields are out of range");
    }
    std::vector<float> pos(3ull * h.n_ant), freq(static_cast<uint64_t>(h.n_shards) * c.shard_channels);
    std::vector<float> extra((h.kind == BF_SERVE_GRID ? 3ull : 4ull) * h.n_beams);
    if (!in.raw(pos.data(), pos.size() * sizeof(float)) || !in.raw(freq.data(), freq.size() * sizeof(float)) ||
        !in.raw(extra.data(), extra.size() * sizeof(float))) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint image is truncated");
    }
    bf_serve_job job{};
    job.kind = static_cast<int32_t>(h.kind);
    job.n_ant = h.n_ant;
    job.n_shards = h.n_shards;
    job.n_beams = h.n_beams;
    job.n_spectra = h.n_spectra;
    job.integration_spectra = h.spectra;
    job.pool_offset = h.pool_offset;
    job.positions = pos.data();
    job.frequencies = freq.data();
    job.directions = h.kind == BF_SERVE_GRID ? extra.data() : nullptr;
    job.trajectories = h.kind == BF_SERVE_GRID ? nullptr : extra.data();
    job.quantize = static_cast<int32_t>(h.quantize);
    Job j;
    BF_RETURN_IF(make_job(s, &job, &j));
    if (h.steps_done > j.n_steps) return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint has more windows than the job");
    const uint64_t rb = regions_bytes(result_regions(c, j.spec, j.lay, h.steps_done));
    if (in.left() != rb) return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint results do not match the job");
    j.resume_step = h.steps_done;
    j.resume_results.resize(rb);
    if (rb > 0 && !in.raw(j.resume_results.data(), rb)) {
        return set_error(BF_ERR_INVALID_ARGUMENT, "checkpoint image is truncated");
    }
    enqueue(s, std::move(j), job_id);
    return BF_OK;
}

BF_API bf_status bf_serve_restore(bf_server* s, const void* image, uint64_t bytes, uint64_t* job_id) {
    try {
        return bf_serve_restore_impl(s, image, bytes, job_id);
    } catch (const std::bad_alloc&) {
        return set_error(BF_ERR_RESOURCE, "host memory exhausted");
    } catch (const std::exception& e) {
        return set_error(BF_ERR_LOGIC, std::string("internal error: ") + e.what());
    }
}

}  // extern "C"
