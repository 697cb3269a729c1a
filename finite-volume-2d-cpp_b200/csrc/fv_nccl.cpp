#include "fv_nccl.h"

#include <dlfcn.h>

#include <cstdlib>
#include <mutex>
#include <type_traits>

namespace fvgpu {

const NcclApi* nccl_api(std::string* err) {
    static std::once_flag once;
    static NcclApi api;
    static bool ok = false;
    static std::string why;
    std::call_once(once, [] {
        // FVGPU_NCCL_LIB names the NCCL library to use: a process that also
        // loads PyTorch must hold PyTorch's own copy, since a second library
        // of the same soname loaded first would stand in for it
        const char* path = std::getenv("FVGPU_NCCL_LIB");
        void* h = nullptr;
        if (path && *path) h = dlopen(path, RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            const char* e = dlerror();
            why = std::string("cannot load libnccl.so.2: ") + (e ? e : "unknown error");
            return;
        }
        bool all = true;
        auto sym = [&](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            if (!fn) {
                all = false;
                why = std::string("libnccl.so.2 lacks ") + name;
            }
        };
        sym(api.GetVersion, "ncclGetVersion");
        sym(api.GetUniqueId, "ncclGetUniqueId");
        sym(api.CommInitRank, "ncclCommInitRank");
        sym(api.CommDestroy, "ncclCommDestroy");
        sym(api.CommAbort, "ncclCommAbort");
        sym(api.CommGetAsyncError, "ncclCommGetAsyncError");
        sym(api.GetErrorString, "ncclGetErrorString");
        sym(api.Send, "ncclSend");
        sym(api.Recv, "ncclRecv");
        sym(api.AllGather, "ncclAllGather");
        sym(api.GroupStart, "ncclGroupStart");
        sym(api.GroupEnd, "ncclGroupEnd");
        ok = all;
    });
    if (!ok) {
        if (err) *err = why;
        return nullptr;
    }
    return &api;
}

}  // namespace fvgpu
