// library.cpp -- app library (kernel-reuse cache) and fused app chains.
//
// The app library restates PfSolve_AppLibrary (PfSolve/pfSolve_AppCollectionManager.hpp:29-148):
// maps from the JW / dgbmv / block keys, ordered lexicographically, to
// initialised applications.  Because every kernel is precompiled here, a hit
// saves the plan work (variant choice, occupancy query), not a compile.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <tuple>

#include "../../include/pfsolve_b200.h"
#include "jw_variants.h"

using namespace pfb;

namespace {
auto tie_key(const PfSolve_MapKey_JonesWorland& k)
{
    return std::make_tuple(k.size[0], k.size[1], k.upperBanded, k.outputBufferStride, k.type);
}
auto tie_key(const PfSolve_MapKey_dgbmv& k)
{
    return std::make_tuple(k.size[0], k.size[1], k.LDA, k.outputBufferStride, k.KU, k.KL);
}
auto tie_key(const PfSolve_MapKey_block& k)
{
    return std::make_tuple(k.size[0], k.size[1], k.inputBufferStride, k.outputBufferStride, k.type, k.lshift);
}
template <class K>
struct KeyLess {
    bool operator()(const K& a, const K& b) const { return tie_key(a) < tie_key(b); }
};
}  // namespace

struct PfSolve_AppLibrary {
    std::map<PfSolve_MapKey_JonesWorland, PfSolveApplication, KeyLess<PfSolve_MapKey_JonesWorland>> jw;
    std::map<PfSolve_MapKey_dgbmv, PfSolveApplication, KeyLess<PfSolve_MapKey_dgbmv>> dgbmv;
    std::map<PfSolve_MapKey_block, PfSolveApplication, KeyLess<PfSolve_MapKey_block>> block;
};

namespace {
template <class Map, class K>
PfSolveResult check(Map& m, const K& key, PfSolveApplication** app)
{
    if (!app) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    auto it = m.find(key);
    *app = (it == m.end()) ? nullptr : &it->second;
    return PFSOLVE_SUCCESS;
}
template <class Map, class K>
PfSolveResult add(Map& m, const K& key, PfSolveApplication* app)
{
    if (!app) return PFSOLVE_ERROR_INVALID_ARGUMENT;
    auto it = m.find(key);
    if (it != m.end() && it->second.internal != app->internal) deletePfSolve(&it->second);
    m[key] = *app;  // the library now owns the plan state (as the reference map copies the app)
    return PFSOLVE_SUCCESS;
}
}  // namespace

extern "C" {

PfSolve_AppLibrary* PfSolveAppLibraryCreate(void) { return new (std::nothrow) PfSolve_AppLibrary(); }

void PfSolveAppLibraryDestroy(PfSolve_AppLibrary* lib)
{
    if (!lib) return;
    for (auto& kv : lib->jw) deletePfSolve(&kv.second);
    for (auto& kv : lib->dgbmv) deletePfSolve(&kv.second);
    for (auto& kv : lib->block) deletePfSolve(&kv.second);
    delete lib;
}

PfSolveResult checkLibrary_JonesWorland(PfSolve_AppLibrary* lib, PfSolve_MapKey_JonesWorland key, PfSolveApplication** app)
{
    return lib ? check(lib->jw, key, app) : PFSOLVE_ERROR_INVALID_ARGUMENT;
}
PfSolveResult addToLibrary_JonesWorland(PfSolve_AppLibrary* lib, PfSolve_MapKey_JonesWorland key, PfSolveApplication* app)
{
    return lib ? add(lib->jw, key, app) : PFSOLVE_ERROR_INVALID_ARGUMENT;
}
PfSolveResult checkLibrary_dgbmv(PfSolve_AppLibrary* lib, PfSolve_MapKey_dgbmv key, PfSolveApplication** app)
{
    return lib ? check(lib->dgbmv, key, app) : PFSOLVE_ERROR_INVALID_ARGUMENT;
}
PfSolveResult addToLibrary_dgbmv(PfSolve_AppLibrary* lib, PfSolve_MapKey_dgbmv key, PfSolveApplication* app)
{
    return lib ? add(lib->dgbmv, key, app) : PFSOLVE_ERROR_INVALID_ARGUMENT;
}
PfSolveResult checkLibrary_block(PfSolve_AppLibrary* lib, PfSolve_MapKey_block key, PfSolveApplication** app)
{
    return lib ? check(lib->block, key, app) : PFSOLVE_ERROR_INVALID_ARGUMENT;
}
PfSolveResult addToLibrary_block(PfSolve_AppLibrary* lib, PfSolve_MapKey_block key, PfSolveApplication* app)
{
    return lib ? add(lib->block, key, app) : PFSOLVE_ERROR_INVALID_ARGUMENT;
}

}  // extern "C"
