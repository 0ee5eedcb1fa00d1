// tuning.cpp -- the run-time configuration table (format in tuning.h).
#include <dlfcn.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "handle.h"
#include "tuning.h"

namespace rsb {
namespace {

struct Entry
{
    int kind; // 0 getrf, 1 vbatched
    char prec;
    int size_max;
    int v[6];
};

struct Table
{
    std::vector<Entry> e; // sorted by (kind, prec, size_max)
};

std::mutex g_mu;
std::shared_ptr<const Table> g_table; // replaced whole; readers copy the pointer
std::once_flag g_default_once;

std::shared_ptr<const Table> current()
{
    std::lock_guard<std::mutex> lk(g_mu);
    return g_table;
}

// Parse the text; false (and nothing changed) on a malformed line.
bool parse(const char* text, Table* out)
{
    std::istringstream in(text);
    std::string line;
    while(std::getline(in, line))
    {
        const size_t hash = line.find('#');
        if(hash != std::string::npos)
            line.resize(hash);
        std::istringstream ls(line);
        std::string kind;
        if(!(ls >> kind))
            continue;
        Entry e{};
        std::string prec;
        int nvals;
        if(kind == "getrf")
        {
            e.kind = 0;
            nvals = 5;
        }
        else if(kind == "vbatched")
        {
            e.kind = 1;
            nvals = 6;
        }
        else
            return false;
        if(!(ls >> prec >> e.size_max) || e.size_max < 1
           || !(prec == "s" || prec == "d" || (prec == "t" && e.kind == 0)))
            return false;
        e.prec = prec[0];
        for(int i = 0; i < nvals; ++i)
            if(!(ls >> e.v[i]) || e.v[i] < 0)
                return false;
        std::string extra;
        if(ls >> extra)
            return false;
        out->e.push_back(e);
    }
    std::sort(out->e.begin(), out->e.end(), [](const Entry& a, const Entry& b) {
        if(a.kind != b.kind)
            return a.kind < b.kind;
        if(a.prec != b.prec)
            return a.prec < b.prec;
        return a.size_max < b.size_max;
    });
    return true;
}

const Entry* find(const Table* t, int kind, char prec, int size)
{
    if(!t)
        return nullptr;
    for(const Entry& e : t->e)
        if(e.kind == kind && e.prec == prec && size <= e.size_max)
            return &e;
    return nullptr;
}

bool read_file(const char* path, std::string* text)
{
    FILE* f = std::fopen(path, "rb");
    if(!f)
        return false;
    char buf[4096];
    size_t k;
    while((k = std::fread(buf, 1, sizeof(buf), f)) > 0)
        text->append(buf, k);
    std::fclose(f);
    return true;
}

rocblas_status install(const char* text)
{
    auto t = std::make_shared<Table>();
    if(!parse(text, t.get()))
        return rocblas_status_invalid_value;
    std::lock_guard<std::mutex> lk(g_mu);
    g_table = std::move(t);
    return rocblas_status_success;
}

void anchor() {}

} // namespace

bool tuned_getrf(char prec, int m, LuCfg* out)
{
    auto t = current();
    const Entry* e = find(t.get(), 0, prec, m);
    if(!e)
        return false;
    *out = LuCfg{e->v[0], e->v[1], e->v[2], e->v[3], e->v[4]};
    return true;
}

bool tuned_vbatched(char prec, int max_n, VbCfg* out)
{
    auto t = current();
    const Entry* e = find(t.get(), 1, prec, max_n);
    if(!e)
        return false;
    *out = VbCfg{e->v[0], e->v[1], e->v[2], e->v[3], e->v[4], e->v[5]};
    return true;
}

void tuning_load_default_once()
{
    std::call_once(g_default_once, [] {
        std::string path;
        const char* env = std::getenv("ROCSOLVER_B200_TUNING");
        if(env && *env)
            path = env;
        else
        {
            Dl_info info;
            if(dladdr(reinterpret_cast<void*>(&anchor), &info) && info.dli_fname)
            {
                path = info.dli_fname;
                const size_t slash = path.rfind('/');
                path = (slash == std::string::npos ? std::string() : path.substr(0, slash + 1))
                       + "tuning_b200.txt";
            }
        }
        std::string text;
        if(!path.empty() && read_file(path.c_str(), &text))
            install(text.c_str());
    });
}

} // namespace rsb

using namespace rsb;

extern "C" ROCSOLVER_EXPORT rocblas_status rocsolver_b200_tuning_set(const char* text)
{
    if(!text)
        return rocblas_status_invalid_pointer;
    tuning_load_default_once(); // a later first handle must not replace this table
    return install(text);
}

extern "C" ROCSOLVER_EXPORT rocblas_status rocsolver_b200_tuning_load(const char* path)
{
    if(!path)
        return rocblas_status_invalid_pointer;
    std::string text;
    if(!read_file(path, &text))
        return rocblas_status_invalid_value;
    return rocsolver_b200_tuning_set(text.c_str());
}

extern "C" ROCSOLVER_EXPORT size_t rocsolver_b200_tuning_get(char* buf, size_t len)
{
    auto t = current();
    std::string s;
    if(t)
        for(const Entry& e : t->e)
        {
            char line[160];
            if(e.kind == 0)
                std::snprintf(line, sizeof(line), "getrf %c %d %d %d %d %d %d\n", e.prec,
                              e.size_max, e.v[0], e.v[1], e.v[2], e.v[3], e.v[4]);
            else
                std::snprintf(line, sizeof(line), "vbatched %c %d %d %d %d %d %d %d\n", e.prec,
                              e.size_max, e.v[0], e.v[1], e.v[2], e.v[3], e.v[4], e.v[5]);
            s += line;
        }
    if(buf && len)
    {
        const size_t k = s.size() < len - 1 ? s.size() : len - 1;
        std::memcpy(buf, s.data(), k);
        buf[k] = '\0';
    }
    return s.size() + 1;
}
