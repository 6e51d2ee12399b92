// refapi.cu -- the reference's public C API (include/cablegen.h) on the B200 engine.
//
// generate() and solve() keep the reference's file contract -- one
// "<sum>.boards" file of sorted u64 per layer (src/generate.c:74-87), one
// "<sum>.tables" file of N keys then N f64 values per layer
// (src/solve.c:29-45) -- and run every layer step on the GPU.  Settings use
// the reference's INI keys, defaults and search path (src/settings.c:34-86,
// inc/external/cfgpath.h:96-135).  Host helpers (arrays, lookup, movedir,
// output_board, string parsing) follow src/array.c, src/solve.c:108-164,
// src/board.c:171-193,395-420 and src/format.c.
#include "cgb_engine.h"
#include "../../include/cablegen.h"
#include "../../include/cablegen_format.h"
#include <algorithm>
#include <cctype>
#include <condition_variable>
#include <deque>
#include <functional>
#include <mutex>
#include <thread>
#include <cerrno>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/resource.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>
#include <vector>

using cgb::u32;
using cgb::u64;

namespace {

// ---- logging (message shapes of the reference's logger) --------------------
enum Level { L_TRACE, L_DBG, L_INFO, L_WARN, L_ERROR };
int g_level = L_INFO;

void logf(Level lv, const char *fmt, ...)
{
    if (lv < g_level) return;
    static const char *tag[] = {"TRACE", "DEBUG", "INFO", "WARN", "ERROR"};
    std::fprintf(stdout, "[%s] ", tag[lv]);
    va_list ap;
    va_start(ap, fmt);
    std::vfprintf(stdout, fmt, ap);
    va_end(ap);
    std::fprintf(stdout, "\n");
    std::fflush(stdout);
}

// ---- settings -----------------------------------------------------------------
// Full settings: min_settings_t first, as the CLI writes through its pointers
// (src/settings.c:30-32, inc/settings.h:15-31).
struct Settings {
    min_settings_t min;
    bool delete_boards;
    bool mask;
    bool compress;
    long long max_prealloc;
    bool use_gpu;
    bool premove;
    long long stsl;
    long long ltc;
    long long smallest_large;
    bool prune;
    bool score;
    bool fp32;  // [Solve] fp32: solve with FP32 tables (library extension, default off)
    // [Generate] checkpoint / resume (library extension, default off): write, after
    // each layer, the state the next layer starts from; start from the newest one
    bool checkpoint;
    bool resume;
};

Settings g_settings = [] {
    Settings s{};
    s.min.free_formation = false;
    s.min.ignore_f = false;
    s.min.cores = 1;
    s.min.nox = 0;
    s.min.bdir = (char *)"./boards/";
    s.min.initial = (char *)"./initial";
    s.min.end_gen = 1200;
    s.min.tdir = (char *)"./tables/";
    s.min.winstates = (char *)"./winstates";
    s.min.end_solve = 0;
    s.min.delete_boards = false;
    s.delete_boards = false;
    s.mask = false;
    s.compress = false;
    s.max_prealloc = 0;
    s.use_gpu = true;
    s.premove = false;
    s.stsl = 200;
    s.ltc = 5;
    s.smallest_large = 6;
    s.prune = false;
    s.score = false;
    s.fp32 = false;
    s.checkpoint = false;
    s.resume = false;
    return s;
}();
bool g_settings_read = false;
bool g_custom_path = false;
std::string g_cfg_path;

// A small INI reader: [section] headers, key = value lines, ';' / '#'
// comments, optional double quotes around a value; section and key names
// compare case-insensitively.
struct Ini {
    struct Entry {
        std::string section, key, value;
    };
    std::vector<Entry> entries;
    static std::string lower(std::string s)
    {
        for (auto &c : s) c = (char)std::tolower((unsigned char)c);
        return s;
    }
    static std::string trim(const std::string &s)
    {
        size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
        return a == std::string::npos ? "" : s.substr(a, b - a + 1);
    }
    bool load(const std::string &path)
    {
        FILE *f = std::fopen(path.c_str(), "rb");
        if (!f) return false;
        std::string section, line;
        char buf[4096];
        while (std::fgets(buf, sizeof buf, f)) {
            line = trim(buf);
            if (line.empty() || line[0] == ';' || line[0] == '#') continue;
            if (line[0] == '[') {
                size_t e = line.find(']');
                section = lower(trim(line.substr(1, e == std::string::npos ? std::string::npos : e - 1)));
                continue;
            }
            size_t eq = line.find('=');
            if (eq == std::string::npos) continue;
            std::string k = lower(trim(line.substr(0, eq))), v = trim(line.substr(eq + 1));
            if (v.size() >= 2 && v.front() == '"' && v.back() == '"') v = v.substr(1, v.size() - 2);
            else {
                size_t c = v.find_first_of(";#");
                if (c != std::string::npos) v = trim(v.substr(0, c));
            }
            entries.push_back({section, k, v});
        }
        std::fclose(f);
        return true;
    }
    const std::string *get(const char *section, const char *key) const
    {
        const std::string s = lower(section), k = lower(key);
        for (const auto &e : entries)
            if (e.section == s && e.key == k) return &e.value;
        return nullptr;
    }
};

std::string default_config_path()
{
    const char *xdg = std::getenv("XDG_CONFIG_HOME");
    if (xdg) return std::string(xdg) + "/cablegen.conf";
    const char *home = std::getenv("HOME");
    if (!home) return "";
    return std::string(home) + "/.config/cablegen.conf";
}

char *dup_str(const std::string &s)
{
    char *p = (char *)std::malloc(s.size() + 1);
    std::memcpy(p, s.c_str(), s.size() + 1);
    return p;
}

void read_settings()
{
    if (g_settings_read) return;
    g_settings_read = true;
    const std::string path = g_custom_path ? g_cfg_path : default_config_path();
    Ini ini;
    if (path.empty() || !ini.load(path)) {
        logf(L_DBG, "No config at %s, using defaults", path.c_str());
        return;
    }
    Settings &s = g_settings;
    auto b = [&](const char *sec, const char *key, bool *out) {
        if (auto v = ini.get(sec, key)) *out = Ini::lower(*v) == "true";
    };
    auto i = [&](const char *sec, const char *key, long long *out) {
        if (auto v = ini.get(sec, key)) *out = std::atoll(v->c_str());
    };
    auto str = [&](const char *sec, const char *key, char **out) {
        if (auto v = ini.get(sec, key)) *out = dup_str(*v);
    };
    b("Cablegen", "free_formation", &s.min.free_formation);
    b("Cablegen", "ignore_f", &s.min.ignore_f);
    i("Cablegen", "cores", &s.min.cores);
    i("Cablegen", "nox", &s.min.nox);
    b("Cablegen", "mask", &s.mask);
    b("Cablegen", "compress", &s.compress);
    i("Cablegen", "max_prealloc", &s.max_prealloc);
    b("Cablegen", "use_gpu", &s.use_gpu);
    b("Generate", "premove", &s.premove);
    str("Generate", "dir", &s.min.bdir);
    str("Generate", "initial", &s.min.initial);
    i("Generate", "end", &s.min.end_gen);
    i("Generate", "stsl", &s.stsl);
    i("Generate", "ltc", &s.ltc);
    i("Generate", "smallest_large", &s.smallest_large);
    b("Generate", "prune", &s.prune);
    b("Generate", "checkpoint", &s.checkpoint);
    b("Generate", "resume", &s.resume);
    str("Solve", "dir", &s.min.tdir);
    str("Solve", "winstates", &s.min.winstates);
    i("Solve", "end", &s.min.end_solve);
    b("Solve", "score", &s.score);
    b("Solve", "delete_boards", &s.delete_boards);
    b("Solve", "fp32", &s.fp32);
}

Settings &settings()
{
    read_settings();
    return g_settings;
}

// ---- host row table, moves, canonical form -----------------------------------
struct HostTable {
    std::vector<unsigned short> move = std::vector<unsigned short>(65536);
    std::vector<u32> ok = std::vector<u32>(2048);
    int ff = -1, ig = -1;
} g_host_table;

void ensure_host_table()
{
    const Settings &s = settings();
    const int ff = s.min.free_formation ? 1 : 0, ig = s.min.ignore_f ? 1 : 0;
    if (g_host_table.ff == ff && g_host_table.ig == ig) return;
    cgb::build_row_table(ff, ig, g_host_table.move.data(), g_host_table.ok.data());
    g_host_table.ff = ff;
    g_host_table.ig = ig;
}

// left move of the four rows; 0 = a row would vacate a 0xf cell, 1 = legal
// but unchanged, 2 = legal and changed
int host_move_left(u64 y, u64 *out)
{
    u64 r = 0;
    bool ok = true, changed = false;
    for (int i = 0; i < 4; i++) {
        const u32 row = (u32)(y >> (16 * i)) & 0xFFFFu;
        const u32 m = g_host_table.move[row];
        ok &= (g_host_table.ok[row >> 5] >> (row & 31)) & 1u;
        changed |= m != row;
        r |= (u64)m << (16 * i);
    }
    *out = r;
    return ok ? 1 + (int)changed : 0;
}

// movedir (src/board.c:171-193): left/right on the rows; up and down rotate
// clockwise, move right / left, and rotate back.  right(x) = H(left(H x)).
bool host_movedir(u64 *b, int d)
{
    ensure_host_table();
    u64 x = *b, m;
    int r;
    switch (d) {
    case right:
        r = host_move_left(cgb::flip_h(x), &m);
        m = cgb::flip_h(m);
        break;
    case up: {
        const u64 t = cgb::rot_cw(x);
        r = host_move_left(cgb::flip_h(t), &m);
        m = cgb::rot_ccw(cgb::flip_h(m));
        break;
    }
    case down: {
        const u64 t = cgb::rot_cw(x);
        r = host_move_left(t, &m);
        m = cgb::rot_ccw(m);
        break;
    }
    default:
        r = host_move_left(x, &m);
        break;
    }
    if (r == 0) return false;  // illegal: board unchanged (src/board.c:163-166)
    *b = m;
    return r == 2;
}

cgb_rules current_rules()
{
    const Settings &s = settings();
    cgb_rules r{};
    r.free_formation = s.min.free_formation;
    r.ignore_f = s.min.ignore_f;
    r.prune = s.prune;
    r.stsl = s.stsl;
    r.ltc = s.ltc;
    r.smallest_large = s.smallest_large;
    r.nox = (int)s.min.nox;
    r.score = s.score;
    return r;
}

bool engine_ready()
{
    cgb::Engine &e = cgb::Engine::get();
    if (!e.ready && !e.init(0)) return false;
    return e.set_rules(current_rules());
}

[[noreturn]] void die(const char *what)
{
    logf(L_ERROR, "%s: %s", what, cgb_last_error());
    std::exit(EXIT_FAILURE);
}

std::string fmt_layer(const char *fmt, long long layer)
{
    int n = std::snprintf(nullptr, 0, fmt, layer);
    std::string s(n > 0 ? n : 0, '\0');
    std::snprintf(&s[0], s.size() + 1, fmt, layer);
    return s;
}

void print_speed(u64 size)
{
    static bool init = false;
    static timespec old;
    timespec now;
    clock_gettime(CLOCK_MONOTONIC, &now);
    if (!init) {
        init = true;
        old = now;
        return;
    }
    const double dt = (now.tv_sec - old.tv_sec) + 1e-9 * (now.tv_nsec - old.tv_nsec);
    old = now;
    if (dt > 0) logf(L_INFO, "Speed: %ld thousand boards per second", (long)((double)size / 1000.0 / dt));
}

bool write_file(const std::string &name, const void *a, u64 na, const void *b, u64 nb)
{
    FILE *f = std::fopen(name.c_str(), "wb");
    if (!f) {
        logf(L_WARN, "Couldn't write to %s!", name.c_str());
        return false;
    }
    bool ok = true;
    if (na) ok &= std::fwrite(a, 1, na, f) == na;
    if (nb) ok &= std::fwrite(b, 1, nb, f) == nb;
    std::fclose(f);
    return ok;
}

// Files are written by one host thread while the GPU goes on with the next
// layers (the reference writes each layer from the layer loop itself,
// src/generate.c:74-87, src/solve.c:29-106).  Each job waits for its
// device-to-host copy (an event on the engine's I/O stream), writes, and hands
// its pinned buffer back; at most `slots` jobs are in flight.
class FileWriter {
  public:
    struct Job {
        cudaEvent_t ready = nullptr;             // the copy into the buffer is complete
        std::function<void()> write;             // runs on the writer thread
        int slot = -1;                           // pinned buffer to hand back
    };
    explicit FileWriter(int slots) : stages_(slots), free_(slots, true)
    {
        cudaGetDevice(&device_);
        thread_ = std::thread([this] { run(); });
    }
    ~FileWriter() { finish(); }
    // a free pinned buffer of at least `bytes` (waits for the writer if none is free)
    int take(u64 bytes, void **p)
    {
        std::unique_lock<std::mutex> lk(m_);
        cv_.wait(lk, [&] { return std::find(free_.begin(), free_.end(), true) != free_.end(); });
        const int i = (int)(std::find(free_.begin(), free_.end(), true) - free_.begin());
        free_[i] = false;
        lk.unlock();
        if (!stages_[i].reserve(bytes + 8)) {
            give_back(i);
            return -1;
        }
        *p = stages_[i].p;
        return i;
    }
    void submit(Job j)
    {
        std::lock_guard<std::mutex> lk(m_);
        jobs_.push_back(std::move(j));
        cv_.notify_all();
    }
    void finish()
    {
        {
            std::lock_guard<std::mutex> lk(m_);
            if (done_) return;
            done_ = true;
            cv_.notify_all();
        }
        thread_.join();
    }

  private:
    std::vector<cgb::HostStage> stages_;
    std::vector<bool> free_;
    std::deque<Job> jobs_;
    std::mutex m_;
    std::condition_variable cv_;
    bool done_ = false;
    int device_ = 0;
    std::thread thread_;

    void give_back(int i)
    {
        std::lock_guard<std::mutex> lk(m_);
        free_[i] = true;
        cv_.notify_all();
    }
    void run()
    {
        cudaSetDevice(device_);
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return done_ || !jobs_.empty(); });
                if (jobs_.empty()) return;
                j = std::move(jobs_.front());
                jobs_.pop_front();
            }
            if (j.ready) {
                CGB_CUDA(cudaEventSynchronize(j.ready));
                cudaEventDestroy(j.ready);
            }
            j.write();
            if (j.slot >= 0) give_back(j.slot);
        }
    }
};

// an event on `main` that `io` waits for, then a copy on `io` and its completion event
cudaEvent_t copy_on_io(void *dst, const void *src, u64 bytes, cudaStream_t main, cudaStream_t io)
{
    cudaEvent_t before = nullptr, after = nullptr;
    if (!CGB_CUDA(cudaEventCreateWithFlags(&before, cudaEventDisableTiming)) ||
        !CGB_CUDA(cudaEventCreateWithFlags(&after, cudaEventDisableTiming)))
        return nullptr;
    bool ok = CGB_CUDA(cudaEventRecord(before, main)) && CGB_CUDA(cudaStreamWaitEvent(io, before, 0)) &&
              (bytes == 0 || CGB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, io))) &&
              CGB_CUDA(cudaEventRecord(after, io));
    cudaEventDestroy(before);
    if (!ok) {
        cudaEventDestroy(after);
        return nullptr;
    }
    return after;
}

// Resume point of a generation: after layer s the engine holds the input set
// of layer s+2 and the 4-spawns of layer s that join layer s+4's input.  A
// checkpoint file "<layer s+2 file>.resume" stores them: four u64 words
// {CKPT_MAGIC, s + 2, |input|, |carry|}, then the two sorted arrays.
constexpr uint64_t CKPT_MAGIC = 0x31454d5553455247ull;  // "GRESUME1"

std::string checkpoint_name(const char *fmt, int next) { return fmt_layer(fmt, next) + ".resume"; }

// layers from the engine go to "<sum>.boards" files through the writer
struct FileSink : cgb::LayerSink {
    const char *fmt = nullptr;
    FileWriter *writer = nullptr;
    bool checkpoint = false;
    std::string last_checkpoint;  // written by the writer thread, removed when superseded
    bool layer(int sum, u64 *d, u64 n, cudaStream_t s, bool *kept) override
    {
        *kept = false;
        cgb::Engine &e = cgb::Engine::get();
        void *h = nullptr;
        const int slot = writer->take(n * 8, &h);
        if (slot < 0) return false;
        // the engine reuses its layer buffer: the copy must be done before the
        // main stream goes on, so it waits for the I/O stream's event
        cudaEvent_t ev = copy_on_io(h, d, n * 8, s, e.io_stream);
        if (!ev || !CGB_CUDA(cudaStreamWaitEvent(s, ev, 0))) return false;
        const std::string f = fmt;
        writer->submit({ev, [h, n, f, sum] {
                            static_arr_info a{true, (uint64_t *)h, (size_t)n};
                            write_boards(a, f.c_str(), sum);
                        },
                        slot});
        if (checkpoint && !write_checkpoint(sum + 2, s)) return false;
        return true;
    }
    bool write_checkpoint(int next, cudaStream_t s)
    {
        cgb::Engine &e = cgb::Engine::get();
        const u64 ns = e.gen.S.n, nc = e.gen.u4.n;
        void *h = nullptr;
        const int slot = writer->take(8 * (4 + ns + nc), &h);
        if (slot < 0) return false;
        uint64_t *w = (uint64_t *)h;
        w[0] = CKPT_MAGIC;
        w[1] = (uint64_t)next;
        w[2] = ns;
        w[3] = nc;
        cudaEvent_t before = nullptr;
        if (!CGB_CUDA(cudaEventCreateWithFlags(&before, cudaEventDisableTiming)) ||
            !CGB_CUDA(cudaEventRecord(before, s)) || !CGB_CUDA(cudaStreamWaitEvent(e.io_stream, before, 0)))
            return false;
        cudaEventDestroy(before);
        if (ns && !CGB_CUDA(cudaMemcpyAsync(w + 4, e.gen.S.p, ns * 8, cudaMemcpyDeviceToHost, e.io_stream)))
            return false;
        cudaEvent_t ev = copy_on_io(w + 4 + ns, e.gen.u4.p, nc * 8, s, e.io_stream);
        if (!ev || !CGB_CUDA(cudaStreamWaitEvent(s, ev, 0))) return false;
        const std::string name = checkpoint_name(fmt, next), prev = last_checkpoint;
        last_checkpoint = name;
        const u64 bytes = 8 * (4 + ns + nc);
        writer->submit({ev, [w, bytes, name, prev] {
                            const std::string tmp = name + ".tmp";
                            if (write_file(tmp, w, bytes, nullptr, 0) && std::rename(tmp.c_str(), name.c_str()) == 0) {
                                if (!prev.empty()) std::remove(prev.c_str());
                            } else {
                                logf(L_WARN, "Couldn't write the checkpoint %s!", name.c_str());
                            }
                        },
                        slot});
        return true;
    }
};

// the newest checkpoint of `fmt` after layer `start` (next = 0 when none; next
// > end when the generation up to `end` is complete)
struct Checkpoint {
    int next = 0;
    std::vector<u64> input, carry;
};
Checkpoint find_checkpoint(const char *fmt, int start, int end)
{
    Checkpoint c;
    for (int next = end + 2; next > start; next -= 2) {
        const std::string name = checkpoint_name(fmt, next);
        FILE *f = std::fopen(name.c_str(), "rb");
        if (!f) continue;
        uint64_t hdr[4];
        bool ok = std::fread(hdr, 8, 4, f) == 4 && hdr[0] == CKPT_MAGIC && hdr[1] == (uint64_t)next;
        if (ok) {
            c.input.resize(hdr[2]);
            c.carry.resize(hdr[3]);
            ok = std::fread(c.input.data(), 8, hdr[2], f) == hdr[2] && std::fread(c.carry.data(), 8, hdr[3], f) == hdr[3];
        }
        std::fclose(f);
        if (ok) {
            c.next = next;
            return c;
        }
        logf(L_WARN, "Ignoring the unreadable checkpoint %s", name.c_str());
        c = Checkpoint{};
    }
    return c;
}

}  // namespace

// =============================================================== C API
extern "C" {

min_settings_t *get_settings_min(void) { return &settings().min; }

void change_config(char *cfg)
{
    if (!cfg || std::strlen(cfg) >= 4096) {
        logf(L_WARN, "Invalid config file location!");
        return;
    }
    g_settings_read = false;  // re-read lazily (src/settings.c:110-120)
    g_custom_path = true;
    g_cfg_path = cfg;
}

void init_settings(void)
{
    settings();
    char buf[4096];
    if (!getcwd(buf, sizeof buf)) {
        logf(L_WARN, "Could not get current working directory!");
        return;
    }
    std::string p = std::string(buf) + "/cablegen.conf";
    change_config(&p[0]);
    settings();
}

char *get_version(void) { return (char *)"cablegen_b200 1.0 (B200 engine)"; }

void generate_lut(void)
{
    ensure_host_table();
}

bool movedir(uint64_t *b, dir d) { return host_movedir(b, (int)d); }

int get_sum(uint64_t b) { return cgb::tile_sum(b); }

double pun_uint64(uint64_t x)
{
    double d;
    std::memcpy(&d, &x, 8);
    return d;
}

void output_board(uint64_t board)
{
    static const char *tiles[16] = {"   ", "2  ", "4  ", "8  ", "16 ", "32 ", "64 ", "128",
                                    "256", "512", "1k ", "2k ", "4k ", "8k ", "m  ", "x  "};
    for (int r = 0; r < 4; r++) {
        for (int c = 0; c < 4; c++) std::printf("%s ", tiles[cgb::tile_at(board, 4 * r + c)]);
        std::printf("\n");
    }
}

// ---- host arrays (src/array.c) -------------------------------------------------
void *malloc_errcheck(size_t size)
{
    void *p = std::malloc(size);
    if (!p) {
        logf(L_ERROR, "Alloc failed!");
        std::exit(EXIT_FAILURE);
    }
    return p;
}

dynamic_arr_info init_darr(bool zero, size_t size)
{
    dynamic_arr_info d;
    d.valid = true;
    d.bp = (uint64_t *)(zero ? std::calloc(size, 8) : std::malloc(8 * size));
    if (!d.bp && size) {
        logf(L_ERROR, "Alloc failed! Download more ram!");
        d.valid = false;
    }
    d.sp = d.bp;
    d.size = size;
    return d;
}

static_arr_info init_sarr(bool zero, size_t size)
{
    static_arr_info s;
    s.valid = true;
    s.bp = (uint64_t *)(zero ? std::calloc(size, 8) : std::malloc(8 * size));
    if (!s.bp && size) {
        logf(L_ERROR, "Alloc failed! Download more ram!");
        s.valid = false;
    }
    s.size = size;
    return s;
}

bool push_back(dynamic_arr_info *a, uint64_t v)
{
    if (!a->valid) return false;
    bool grew = false;
    if (!a->bp || a->sp == a->bp + a->size) {
        const size_t used = a->bp ? (size_t)(a->sp - a->bp) : 0;
        const size_t cap = a->size ? a->size * 3 : 1;  // x3 growth (REALLOC_MULT)
        uint64_t *p = (uint64_t *)std::realloc(a->bp, cap * 8);
        if (!p) {
            logf(L_ERROR, "Alloc failed! Download more ram!");
            a->valid = false;
            return false;
        }
        a->bp = p;
        a->sp = p + used;
        a->size = cap;
        grew = true;
    }
    *(a->sp++) = v;
    return grew;
}

static_arr_info shrink_darr(dynamic_arr_info *a)
{
    if (!a->valid) return static_arr_info{false, a->bp, (size_t)(a->sp - a->bp)};
    a->valid = false;
    const size_t n = a->bp ? (size_t)(a->sp - a->bp) : 0;
    if (n == 0) {
        std::free(a->bp);
        a->bp = a->sp = nullptr;
        a->size = 0;
        return static_arr_info{true, nullptr, 0};
    }
    uint64_t *p = (uint64_t *)std::realloc(a->bp, n * 8);
    if (!p) return static_arr_info{false, a->bp, n};
    return static_arr_info{true, p, n};
}

dynamic_arr_info concat(dynamic_arr_info *a, dynamic_arr_info *b)
{
    if (!a->valid || !b->valid) {
        logf(L_WARN, "Refusing to concatenate invalid arrays!");
        return *a;
    }
    a->valid = b->valid = false;
    const size_t na = a->sp - a->bp, nb = b->sp - b->bp;
    dynamic_arr_info r{true, nullptr, nullptr, na + nb};
    if (a->size >= na + nb) {
        r.bp = a->bp;
    } else {
        r.bp = (uint64_t *)malloc_errcheck((na + nb) * 8 + 8);
        if (na) std::memcpy(r.bp, a->bp, na * 8);
        std::free(a->bp);
    }
    if (nb) std::memcpy(r.bp + na, b->bp, nb * 8);
    std::free(b->bp);
    r.sp = r.bp + na + nb;
    return r;
}

void destroy_darr(dynamic_arr_info *a)
{
    std::free(a->bp);
    a->valid = false;
}

void destroy_sarr(static_arr_info *a)
{
    std::free(a->bp);
    a->valid = false;
}

// ---- files ---------------------------------------------------------------------
void write_boards(const static_arr_info n, const char *fmt, const int layer)
{
    const std::string name = fmt_layer(fmt, layer);
    logf(L_INFO, "Writing %lu boards to %s (%lu bytes)", (unsigned long)n.size, name.c_str(),
         (unsigned long)(8 * n.size));
    write_file(name, n.bp, 8 * n.size, nullptr, 0);
    print_speed(n.size);
}

static_arr_info read_boards(const char *path)
{
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        logf(L_WARN, "Couldn't read %s!", path);
        return static_arr_info{false, nullptr, 0};
    }
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::rewind(f);
    if (sz % 8 != 0) logf(L_WARN, "sz %%8 != 0, this is probably not a real table!");
    uint64_t *data = (uint64_t *)malloc_errcheck(sz > 0 ? sz : 1);
    if ((long)std::fread(data, 1, sz, f) != sz) {
        std::fclose(f);
        std::free(data);
        logf(L_WARN, "Couldn't read %s!", path);
        return static_arr_info{false, nullptr, 0};
    }
    std::fclose(f);
    logf(L_INFO, "Read %ld bytes (%ld boards) from %s", sz, sz / 8, path);
    return static_arr_info{true, data, (size_t)(sz / 8)};
}

void read_boards2(static_arr_info *b, const char *path) { *b = read_boards(path); }

void read_table(table *t, const char *path)
{
    FILE *f = std::fopen(path, "rb");
    t->key = init_sarr(false, 0);
    t->value = init_sarr(false, 0);
    if (!f) {
        logf(L_WARN, "Couldn't read %s!", path);
        t->key.valid = t->value.valid = false;
        return;
    }
    std::fseek(f, 0, SEEK_END);
    const long sz = std::ftell(f);
    std::rewind(f);
    if (sz % 16 != 0) logf(L_WARN, "sz %%16 != 0, this is probably not a real table!");
    const size_t n = sz / 16;
    std::free(t->key.bp);
    std::free(t->value.bp);
    t->key = init_sarr(false, n);
    t->value = init_sarr(false, n);
    if (std::fread(t->key.bp, 8, n, f) != n || std::fread(t->value.bp, 8, n, f) != n) {
        logf(L_WARN, "Error reading file!");
        t->key.valid = t->value.valid = false;
    } else {
        logf(L_INFO, "Read %ld bytes (%ld boards) from %s", sz, (long)n, path);
    }
    std::fclose(f);
}

// solve.c:108-164: exact membership; a miss or an empty table gives 0.0
double lookup(uint64_t key, table *t, bool canonicalize)
{
    if (t->key.size == 0) return 0.0;
    if (canonicalize) key = cgb::canonical(key);
    const uint64_t *b = t->key.bp, *e = b + t->key.size;
    const uint64_t *it = std::lower_bound(b, e, key);
    if (it == e || *it != key) return 0.0;
    return pun_uint64(t->value.bp[it - b]);
}

// ---- generation (src/generate.c:551-615) -----------------------------------------
void generate(const int start, const int end, const char *fmt, const static_arr_info *initial)
{
    Settings &s = settings();
    generate_lut();
    if (s.premove) logf(L_WARN, "premove is not supported (the reference's premove path is broken); ignoring it");
    if (!engine_ready()) die("generate: GPU engine");
    FileWriter writer(3);
    FileSink sink;
    sink.fmt = fmt;
    sink.writer = &writer;
    sink.checkpoint = s.checkpoint;
    cgb::GenTimes tm;
    Checkpoint ck;
    if (s.resume) ck = find_checkpoint(fmt, start, end);
    bool ok = true;
    if (ck.next > end) {
        logf(L_INFO, "%s: every layer up to %d is already generated", checkpoint_name(fmt, ck.next).c_str(), end);
    } else if (ck.next) {
        logf(L_INFO, "Resuming at layer %d from %s", ck.next, checkpoint_name(fmt, ck.next).c_str());
        sink.last_checkpoint = checkpoint_name(fmt, ck.next);
        ok = cgb::Engine::get().generate(ck.input.data(), ck.input.size(), ck.next, end, sink, &tm, ck.carry.data(),
                                         ck.carry.size());
    } else {
        ok = cgb::Engine::get().generate(initial->bp, initial->size, start, end, sink, &tm);
    }
    writer.finish();
    if (!ok) die("generate");
    rusage ru;
    if (getrusage(RUSAGE_SELF, &ru) == 0) logf(L_INFO, "Peak host RSS:  %.2f MiB", ru.ru_maxrss / 1024.0);
}

// ---- solve (src/solve.c:172-224) ---------------------------------------------------
void solve(unsigned start, unsigned end, char *posfmt, char *tablefmt, const static_arr_info *winstates)
{
    Settings &s = settings();
    generate_lut();
    if (!engine_ready()) die("solve: GPU engine");
    cgb::Engine &e = cgb::Engine::get();
    cudaStream_t st = e.stream;
    const int vb = s.fp32 ? 4 : 8;
    std::vector<u64> ws = cgb::expand_winstates(winstates->bp, (int)winstates->size);
    u64 *d_ws = nullptr;
    if (!cgb::dev_alloc((void **)&d_ws, ws.size() * 8 + 8, st)) die("solve");
    if (!ws.empty() && !CGB_CUDA(cudaMemcpyAsync(d_ws, ws.data(), ws.size() * 8, cudaMemcpyHostToDevice, st)))
        die("solve");
    const cgb::SolveRules rules = cgb::make_solve_rules(current_rules(), d_ws, (int)ws.size());
    struct Lay {
        u64 *keys = nullptr;
        void *vals = nullptr;
        u64 n = 0;
        cgb::IndexStorage store;
        cgb::LayerIndex ix;
    };
    Lay t2, t4, cur;
    FileWriter writer(3);
    cgb::CanonPlan plan;
    bool have_plan = false;
    for (unsigned i = start; i >= end && i; i -= 2) {
        const std::string bname = fmt_layer(posfmt, i);
        static_arr_info keys = read_boards(bname.c_str());
        if (s.delete_boards) std::remove(bname.c_str());
        cur = Lay{};
        cur.n = keys.valid ? keys.size : 0;
        if (!cgb::dev_alloc((void **)&cur.keys, cur.n * 8 + 8, st) || !cgb::dev_alloc(&cur.vals, cur.n * vb + 8, st))
            die("solve");
        if (cur.n && !CGB_CUDA(cudaMemcpyAsync(cur.keys, keys.bp, cur.n * 8, cudaMemcpyHostToDevice, st)))
            die("solve");
        // the images that can be canonical follow the 0xf mask of the layer's boards
        if (!have_plan && cur.n) {
            plan = cgb::make_canon_plan(keys.bp[0], current_rules().free_formation != 0);
            have_plan = true;
        }
        const bool ok = vb == 4 ? cgb::solve_layer_f32(cur.keys, cur.n, (float *)cur.vals, t2.ix, t4.ix, rules, e.rt,
                                                        e.ctr, st, plan)
                                : cgb::solve_layer_f64(cur.keys, cur.n, (double *)cur.vals, t2.ix, t4.ix, rules, e.rt,
                                                        e.ctr, st, plan);
        if (!ok) die("solve");
        // the values go to a pinned buffer on the I/O stream; the writer thread
        // writes the table (keys from the .boards file, values widened to f64
        // for FP32 tables, as the file format demands) while the next layer runs
        void *h = nullptr;
        const int slot = writer.take(cur.n * vb, &h);
        if (slot < 0) die("solve");
        // copies of the earlier layers (t4's values among them) end at this
        // event; the copy of this layer's values, enqueued next, is not waited for
        cudaEvent_t earlier_io = nullptr;
        if (!CGB_CUDA(cudaEventCreateWithFlags(&earlier_io, cudaEventDisableTiming)) ||
            !CGB_CUDA(cudaEventRecord(earlier_io, e.io_stream)))
            die("solve");
        cudaEvent_t ev = copy_on_io(h, cur.vals, cur.n * vb, st, e.io_stream);
        if (!ev) die("solve");
        const std::string tname = fmt_layer(tablefmt, i);
        const u64 n = cur.n;
        writer.submit({ev, [tname, keys, h, n, vb] {
                           const void *vals = h;
                           std::vector<double> widened;
                           if (vb == 4) {
                               widened.resize(n);
                               for (u64 k = 0; k < n; k++) widened[k] = ((const float *)h)[k];
                               vals = widened.data();
                           }
                           logf(L_INFO, "Writing %lu boards to %s (%lu bytes)", (unsigned long)n, tname.c_str(),
                                (unsigned long)(16 * n));
                           write_file(tname, keys.bp, 8 * n, vals, 8 * n);
                           print_speed(n);
                           std::free(keys.bp);
                       },
                       slot});
        cur.ix.keys = cur.keys;
        cur.ix.vals = cur.vals;
        cur.ix.n = cur.n;
        if (!cgb::build_index(cur.ix, e.index_kind, vb, cur.store, e.bucket_bits, e.ctr, st)) die("solve");
        // the I/O stream may still read t4's values (copied two layers ago)
        if (!CGB_CUDA(cudaStreamWaitEvent(st, earlier_io, 0))) die("solve");
        cudaEventDestroy(earlier_io);
        for (void *p : {(void *)t4.keys, t4.vals, t4.store.p}) cgb::dev_free(p, st);
        t4 = t2;
        t2 = cur;
    }
    writer.finish();
    for (Lay *x : {&t2, &t4})
        for (void *p : {(void *)x->keys, x->vals, x->store.p}) cgb::dev_free(p, st);
    cgb::dev_free(d_ws, st);
    cudaStreamSynchronize(st);
}

// ---- self-test (src/test.c:366-385) ----------------------------------------------
// Known answers of the reference's own test(): lookup of keys 0..99 holding
// 99-i, array growth and concatenation, duplicate removal (here through the
// GPU sort + unique), symmetry orbits and canonical invariance, tile
// detection, bit macros, don't-care pattern matching, and a short generation
// run to /dev/null.
bool test(void)
{
    bool ok = true;
    auto fail = [&](const char *what) {
        logf(L_ERROR, "%s failed!", what);
        ok = false;
    };
    logf(L_INFO, "Testing searching");
    {
        table t;
        t.key = init_sarr(false, 100);
        t.value = init_sarr(false, 100);
        for (int i = 0; i < 100; i++) {
            const double v = 99 - i;
            t.key.bp[i] = i;
            std::memcpy(&t.value.bp[i], &v, 8);
        }
        for (int i = 0; i < 100; i++)
            if (lookup((uint64_t)i, &t, false) != (double)(99 - i)) fail("Search test");
        if (lookup(1000, &t, false) != 0.0) fail("Search miss test");
        std::free(t.key.bp);
        std::free(t.value.bp);
    }
    logf(L_INFO, "Testing dynamic arrays");
    for (size_t n = 0; n < 50 && ok; n++)
        for (size_t m = 0; m < 50; m++) {
            dynamic_arr_info a = init_darr(false, n), b = init_darr(false, m);
            for (size_t i = 0; i < n; i++) push_back(&a, i);
            for (size_t i = 0; i < m; i++) push_back(&b, i);
            dynamic_arr_info c = concat(&a, &b);
            if ((size_t)(c.sp - c.bp) != n + m) fail("Concatenation test");
            for (size_t i = 0; i < n + m && ok; i++)
                if (c.bp[i] != (i < n ? i : i - n)) fail("Concatenation test");
            std::free(c.bp);
            if (!ok) break;
        }
    logf(L_INFO, "Testing deduplication on the GPU");
    if (engine_ready()) {
        const uint64_t in[6] = {2, 5, 6, 5, 4, 5};
        uint64_t *d = nullptr, *d2 = nullptr, *d3 = nullptr;
        u64 cnt = 0;
        int in_tmp = 0, passes = 0;
        cudaMalloc(&d, 64);
        cudaMalloc(&d2, 64);
        cudaMalloc(&d3, 64);
        cudaMemcpy(d, in, sizeof in, cudaMemcpyHostToDevice);
        if (cgb_sort(d, d2, 6, &in_tmp, &passes) != 0 || cgb_unique(in_tmp ? d2 : d, 6, d3, &cnt) != 0) {
            fail("Deduplication (device error)");
        } else {
            uint64_t out[6] = {0};
            cudaMemcpy(out, d3, cnt * 8, cudaMemcpyDeviceToHost);
            const uint64_t want[4] = {2, 4, 5, 6};
            if (cnt != 4 || std::memcmp(out, want, sizeof want) != 0) fail("Deduplication test");
        }
        cudaFree(d);
        cudaFree(d2);
        cudaFree(d3);
    } else {
        fail("GPU engine");
    }
    logf(L_INFO, "Testing symmetry generation and canonicalization");
    {
        uint64_t x = 0x123456789ABCDEFull;
        for (int it = 0; it < 10000 && ok; it++) {
            x ^= x << 13;
            x ^= x >> 7;
            x ^= x << 17;
            const uint64_t b = x & 0x7777777777777777ull;  // no 0xe/0xf: distinct images
            const std::vector<u64> im = cgb::expand_winstates(&b, 1);
            for (u64 a : im) {
                if (get_sum(a) != get_sum(b)) fail("Symmetry sum test");
                if (cgb::canonical(a) != cgb::canonical(b)) fail("Canonicalization test");
            }
        }
    }
    logf(L_INFO, "Testing tile detection");
    for (int v = 0; v < 16; v++) {
        const uint64_t b = 0x0123456789ABCDEFull;
        bool naive = false;
        for (int c = 0; c < 16; c++) naive |= GET_TILE(b, c) == v;
        if (naive != cgb::has_tile(b, v)) fail("Tile detection test");
    }
    logf(L_INFO, "Testing bit operations");
    {
        uint16_t t = 0;
        for (int i = 0; i < 16; i++) {
            SETBIT(t, i);
            for (int j = 0; j <= i; j++)
                if (!GETBIT(t, j)) fail("Bit test");
        }
        for (int i = 0; i < 16; i++) {
            CLEARBIT(t, i);
            if (GETBIT(t, i)) fail("Bit test");
        }
    }
    logf(L_INFO, "Checking settings (accuracy not checked, verify manually)");
    {
        const Settings &st = settings();
        logf(L_INFO, ".free_formation %d", st.min.free_formation);
        logf(L_INFO, ".ignore_f %d", st.min.ignore_f);
        logf(L_INFO, ".cores %lld", st.min.cores);
        logf(L_INFO, ".nox %lld", st.min.nox);
        logf(L_INFO, ".bdir %s", st.min.bdir);
        logf(L_INFO, ".end_gen %lld", st.min.end_gen);
        logf(L_INFO, ".stsl %lld .ltc %lld .smallest_large %lld .prune %d", st.stsl, st.ltc, st.smallest_large,
             st.prune);
        logf(L_INFO, ".tdir %s .end_solve %lld .score %d", st.min.tdir, st.min.end_solve, st.score);
    }
    logf(L_INFO, "Testing comparison");
    {
        uint64_t pat = 0, x = 88172645463325252ull;
        for (int it = 0; it < 10000; it++) {
            x ^= x << 13;
            x ^= x >> 7;
            x ^= x << 17;
            if (!cgb::matches(x, pat)) fail("Comparison test");
            const int cell = (int)(x >> 60);
            SET_TILE(pat, cell, GET_TILE(x, cell));
            if (!cgb::matches(x, pat)) fail("Comparison test");
            SET_TILE(pat, cell, 0);
        }
    }
    logf(L_INFO, "Testing generation (correctness not checked).");
    {
        uint64_t b = 0x1000002000000000ull;
        static_arr_info a{true, &b, 1};
        generate(get_sum(b), get_sum(b) + 16, "/dev/null", &a);
        logf(L_INFO, "Done testing generation.");
    }
    if (!ok) {
        logf(L_ERROR, "One or more tests failed!");
        std::exit(EXIT_FAILURE);
    }
    logf(L_INFO, "All tests passed!");
    return ok;
}

// ---- string helpers (src/format.c) ------------------------------------------------
char *format_str(const char *fmt, ...)
{
    va_list a, b;
    va_start(a, fmt);
    va_copy(b, a);
    const int n = std::vsnprintf(nullptr, 0, fmt, a);
    va_end(a);
    char *buf = (char *)malloc_errcheck((size_t)(n > 0 ? n : 0) + 1);
    std::vsnprintf(buf, (size_t)(n > 0 ? n : 0) + 1, fmt, b);
    va_end(b);
    return buf;
}

bool isdigit_radix(const char input, const unsigned int radix)
{
    int v = -1;
    if (input >= '0' && input <= '9') v = input - '0';
    else if (std::isalpha((unsigned char)input)) v = std::tolower((unsigned char)input) - 'a' + 10;
    return v >= 0 && (unsigned)v < radix;
}

atoi_res safe_atoi(const char *input)
{
    atoi_res r{0, 0};
    errno = 0;
    r.res = std::strtol(input, nullptr, 10);
    if (r.res == LONG_MAX || r.res == LONG_MIN) r.status = ERANGE;
    else if (errno) r.status = errno;
    else if (!r.res)
        for (const char *c = input; *c; c++)
            if (!std::isspace((unsigned char)*c) && !std::isdigit((unsigned char)*c)) r.status = EINVAL;
    errno = 0;
    return r;
}

atoi_res_ll safe_atoi_ll(const char *input, const int radix)
{
    atoi_res_ll r{0, 0};
    if (radix < 2 || radix > 36) {
        r.status = EINVAL;
        return r;
    }
    errno = 0;
    r.res = std::strtoll(input, nullptr, radix);
    if (r.res == LLONG_MAX || r.res == LLONG_MIN) r.status = ERANGE;
    else if (errno) r.status = errno;
    else if (!r.res)
        for (const char *c = input; *c; c++)
            if (!std::isspace((unsigned char)*c) && !isdigit_radix(*c, radix)) r.status = EINVAL;
    errno = 0;
    return r;
}

}  // extern "C"
