// logger.cpp -- the logging session behind logger.h and the rocsolver_log_* C API
// (reference: library/src/common/rocsolver_logger.cpp, library/include/rocsolver/
// rocsolver-functions.h:66-119).
#include "logger.h"

#include <cuda_runtime.h>
#include <errno.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>

#include <atomic>
#include <chrono>
#include <map>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "handle.h"

namespace rsb {
namespace logging {
namespace {

struct Frame
{
    std::string name;   // logged name (rocsolver_dgetrf_strided_batched, rocsolver_getrf_template)
    int level;
    double start_us;
};

struct Prof
{
    int level = 0;
    long calls = 0;
    double us = 0;
    std::map<std::string, Prof> nested;
};

struct Session
{
    uint32_t mode = 0;
    int max_levels = 1;
    FILE* trace = stderr;
    FILE* bench = stderr;
    FILE* profile = stderr;
    std::map<std::string, FILE*> files;   // one FILE per distinct path
    std::unordered_map<rocblas_handle, std::vector<Frame>> stacks;
    std::unordered_map<rocblas_handle, std::string> trace_buf;
    std::map<std::string, Prof> prof;
};

std::mutex g_mu;
Session* g_session = nullptr;
std::atomic<uint32_t> g_mode{0};
thread_local rocblas_handle t_current = nullptr;
thread_local int t_depth = 0;

double now_us()
{
    using namespace std::chrono;
    return duration<double, std::micro>(steady_clock::now().time_since_epoch()).count();
}

FILE* open_stream(Session* s, const char* env)
{
    const char* path = getenv(env);
    if(!path)
        path = getenv("ROCSOLVER_LOG_PATH");
    if(!path)
        return stderr;
    auto it = s->files.find(path);
    if(it != s->files.end())
        return it->second;
    FILE* f = fopen(path, "w");
    if(!f)
        return nullptr;
    char ver[64] = {0};
    rocsolver_get_version_string(ver, sizeof(ver));
    fprintf(f, "ROCSOLVER LOG FILE\nrocSOLVER Version: %s\nrocBLAS Version: none (B200 build)\n",
            ver);
    fflush(f);
    s->files[path] = f;
    return f;
}

std::string pairs(std::initializer_list<Arg> args, const char* kv_sep, const char* sep)
{
    std::string out;
    bool first = true;
    for(const Arg& a : args)
    {
        if(!first)
            out += sep;
        first = false;
        out += a.key;
        out += kv_sep;
        out += a.val;
    }
    return out;
}

void write_profile(Session* s, std::string& out, const std::map<std::string, Prof>& m)
{
    for(const auto& kv : m)
    {
        const Prof& p = kv.second;
        char line[512];
        snprintf(line, sizeof(line), "%*s%s: Calls: %ld, Total Time: %.3f ms",
                 4 * (p.level > 0 ? p.level - 1 : 0), "", kv.first.c_str(), p.calls,
                 p.us * 1e-3);
        out += line;
        if(!p.nested.empty())
        {
            double in = 0;
            for(const auto& c : p.nested)
                in += c.second.us;
            snprintf(line, sizeof(line), " (in nested functions: %.3f ms)\n", in * 1e-3);
            out += line;
            if(p.level < s->max_levels)
                write_profile(s, out, p.nested);
        }
        else
            out += "\n";
    }
}

void print_profile(Session* s, bool clear)
{
    if(!(s->mode & PROFILE) || s->prof.empty())
        return;
    std::string out;
    write_profile(s, out, s->prof);
    fprintf(s->profile, "------- PROFILE -------\n%s\n", out.c_str());
    fflush(s->profile);
    if(clear)
        s->prof.clear();
}

bool parse_env(const char* name, long lo, long hi, long* out)
{
    const char* v = getenv(name);
    if(!v)
        return true;
    errno = 0;
    char* end = nullptr;
    const long x = strtol(v, &end, 0);
    if(errno || end == v || x < lo || x > hi)
        return false;
    *out = x;
    return true;
}

} // namespace

uint32_t mode() { return g_mode.load(std::memory_order_relaxed); }

rocblas_handle current() { return t_current; }

Scope::Scope(rocblas_handle h, char prec, const char* name, std::initializer_list<Arg> args,
             bool top)
    : handle_(h), top_(top), active_(false)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Session* s = g_session;
    if(!s)
        return;
    std::vector<Frame>& st = s->stacks[h];
    Frame f;
    f.level = (int)st.size();
    f.name = top ? std::string("rocsolver_") + (prec ? std::string(1, prec) : std::string())
                       + name
                 : std::string(name);
    if(!top && f.name.rfind("rocsolver_", 0) != 0 && f.name.find("kernel") == std::string::npos)
        f.name = "rocsolver_" + f.name + "_template";
    f.start_us = now_us();
    if(top)
    {
        if(s->mode & BENCH)
        {
            fprintf(s->bench, "./rocsolver-bench -f %s -r %c %s\n", name, prec ? prec : 'd',
                    pairs(args, " ", " ").c_str());
            fflush(s->bench);
        }
        if(s->mode & TRACE)
            s->trace_buf[h] += "------- ENTER " + f.name + " trace tree -------\n";
        t_current = h;
    }
    else if((s->mode & TRACE) && f.level <= s->max_levels)
    {
        std::string line(4 * (f.level > 0 ? f.level - 1 : 0), ' ');
        line += f.name;
        if(args.size())
            line += " (" + pairs(args, " ", ", ") + ")";
        s->trace_buf[h] += line + "\n";
    }
    st.push_back(std::move(f));
    ++t_depth;
    active_ = true;
}

Scope::~Scope()
{
    if(!active_)
        return;
    cudaStream_t stream = handle_ ? handle_->stream : nullptr;
    bool sync = false;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        sync = g_session && (g_session->mode & PROFILE) && handle_ && !top_;
    }
    // profile timing waits for the call's work (outside the lock)
    if(sync)
        cudaStreamSynchronize(stream);
    const double t = now_us();
    std::lock_guard<std::mutex> lk(g_mu);
    --t_depth;
    if(top_ && t_depth == 0)
        t_current = nullptr;
    Session* s = g_session;
    if(!s)
        return;
    auto sit = s->stacks.find(handle_);
    if(sit == s->stacks.end() || sit->second.empty())
        return;
    std::vector<Frame>& st = sit->second;
    Frame f = st.back();
    st.pop_back();
    // profile: nested steps only, keyed by their callers below the entry point (as the
    // reference's profile log records template-level and kernel calls)
    if((s->mode & PROFILE) && !top_)
    {
        std::map<std::string, Prof>* m = &s->prof;
        for(size_t i = 1; i < st.size(); ++i)
            m = &(*m)[st[i].name].nested;
        Prof& p = (*m)[f.name];
        p.level = f.level;
        p.calls += 1;
        p.us += t - f.start_us;
    }
    if(top_ && (s->mode & TRACE))
    {
        std::string& buf = s->trace_buf[handle_];
        buf += "------- EXIT " + f.name + " trace tree -------\n\n";
        fputs(buf.c_str(), s->trace);
        fflush(s->trace);
        buf.clear();
    }
    if(st.empty())
    {
        s->stacks.erase(sit);
        s->trace_buf.erase(handle_);
    }
}

} // namespace logging
} // namespace rsb

using namespace rsb::logging;

extern "C" {

rocblas_status rocsolver_log_begin(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if(g_session)
        return rocblas_status_internal_error;
    std::unique_ptr<Session> s(new Session());
    long layer = 0, levels = 1;
    if(!parse_env("ROCSOLVER_LAYER", 0, (long)UINT32_MAX, &layer)
       || !parse_env("ROCSOLVER_LEVELS", 1, INT_MAX, &levels))
        return rocblas_status_internal_error;
    s->mode = (uint32_t)layer;
    s->max_levels = (int)levels;
    s->trace = open_stream(s.get(), "ROCSOLVER_LOG_TRACE_PATH");
    s->bench = open_stream(s.get(), "ROCSOLVER_LOG_BENCH_PATH");
    s->profile = open_stream(s.get(), "ROCSOLVER_LOG_PROFILE_PATH");
    if(!s->trace || !s->bench || !s->profile)
    {
        for(auto& kv : s->files)
            fclose(kv.second);
        return rocblas_status_internal_error;
    }
    g_session = s.release();
    g_mode.store(g_session->mode, std::memory_order_relaxed);
    return rocblas_status_success;
}

rocblas_status rocsolver_log_end(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    Session* s = g_session;
    if(!s || !s->stacks.empty())
        return rocblas_status_internal_error;
    print_profile(s, false);
    for(auto& kv : s->files)
        fclose(kv.second);
    g_mode.store(0, std::memory_order_relaxed);
    g_session = nullptr;
    delete s;
    return rocblas_status_success;
}

rocblas_status rocsolver_log_set_layer_mode(const rocblas_layer_mode_flags layer_mode)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if(!g_session)
        return rocblas_status_internal_error;
    g_session->mode = layer_mode;
    g_mode.store(layer_mode, std::memory_order_relaxed);
    return rocblas_status_success;
}

rocblas_status rocsolver_log_set_max_levels(const rocblas_int max_levels)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if(!g_session)
        return rocblas_status_internal_error;
    if(max_levels < 1)
        return rocblas_status_invalid_value;
    g_session->max_levels = max_levels;
    return rocblas_status_success;
}

rocblas_status rocsolver_log_restore_defaults(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if(!g_session)
        return rocblas_status_internal_error;
    g_session->mode = 0;
    g_session->max_levels = 1;
    g_mode.store(0, std::memory_order_relaxed);
    return rocblas_status_success;
}

rocblas_status rocsolver_log_write_profile(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if(!g_session)
        return rocblas_status_internal_error;
    print_profile(g_session, false);
    return rocblas_status_success;
}

rocblas_status rocsolver_log_flush_profile(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if(!g_session)
        return rocblas_status_internal_error;
    print_profile(g_session, true);
    return rocblas_status_success;
}

} // extern "C"
