// NCCL entry points of a domain decomposition's exchanges, resolved at run
// time (the library named by the FVGPU_NCCL_LIB environment variable, else
// libnccl.so.2: the copy the process has already loaded, else the system's),
// so that the library itself loads and runs single-part solves without NCCL.
#pragma once
#include <nccl.h>

#include <string>

namespace fvgpu {

struct NcclApi {
    ncclResult_t (*GetVersion)(int*);
    ncclResult_t (*GetUniqueId)(ncclUniqueId*);
    ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int);
    ncclResult_t (*CommDestroy)(ncclComm_t);
    ncclResult_t (*CommAbort)(ncclComm_t);
    ncclResult_t (*CommGetAsyncError)(ncclComm_t, ncclResult_t*);
    const char* (*GetErrorString)(ncclResult_t);
    ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*AllGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t);
    ncclResult_t (*GroupStart)();
    ncclResult_t (*GroupEnd)();
};

// The loaded API, or nullptr with the reason in *err.
const NcclApi* nccl_api(std::string* err);

}  // namespace fvgpu
