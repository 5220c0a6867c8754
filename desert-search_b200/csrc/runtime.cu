// Library runtime: error strings, device selection (dsg_init), shared state.
#include "common.cuh"
#include <cstdarg>
#include <mutex>
#include <stdexcept>

namespace dsg {
namespace {
thread_local char g_err[512] = "";
DeviceInfo g_dev;
std::mutex g_init_mu;
}
void set_error(const char *fmt, ...) {
    va_list ap; va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}
const DeviceInfo &device_info() { return g_dev; }
void require_init() {
    if (g_dev.device < 0) { set_error("dsg_init has not been called"); throw std::runtime_error("dsg_init has not been called"); }
    DSG_CU(cudaSetDevice(g_dev.device));
}
void world_upload(int device);        // world.cpp
void proxy_set_cut(float cut);        // proxy.cu
void proxy32_set_cut(float cut);      // proxy_f32.cu
}  // namespace dsg

extern "C" const char *dsg_last_error(void) { return dsg::g_err; }

extern "C" int dsg_init(int device, float cut) {
    return dsg::guarded([&] {
        std::lock_guard<std::mutex> l(dsg::g_init_mu);
        int n = 0;
        DSG_CU(cudaGetDeviceCount(&n));
        DSG_ARG(device >= 0 && device < n, "dsg_init: no such device");
        DSG_CU(cudaSetDevice(device));
        if (dsg::g_dev.device != device) {
            cudaDeviceProp p;
            DSG_CU(cudaGetDeviceProperties(&p, device));
            DSG_ARG(p.major == 10, "dsg_init: libdsgpu is built for sm_100a (B200) only");
            dsg::g_dev.sms = p.multiProcessorCount;
            DSG_CU(cudaDeviceGetAttribute(&dsg::g_dev.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
            dsg::world_upload(device);
            dsg::g_dev.device = device;
        }
        dsg::proxy_set_cut(cut);
        dsg::proxy32_set_cut(cut);
        return DSG_OK;
    });
}
