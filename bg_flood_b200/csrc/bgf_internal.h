// Internal declarations shared by the C-ABI layer and the kernel launchers.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace bgf {

struct TimeState;
struct SegDev;
template <class T> struct DevModel;
template <class T> struct StepParams;

// Kernel launchers, built twice (bgf_flow.cu): "exact" reproduces the reference
// CPU arithmetic bit for bit, "fast" trades the last bits for speed.
#define BGF_DECLARE_LAUNCHERS                                                                                   \
    template <class T> cudaError_t configure_kernels();                                                        \
    template <class T>                                                                                         \
    void launch_flux(const DevModel<T>& m, const StepParams<T>& p, int engine, int parity, cudaStream_t st);   \
    template <class T>                                                                                         \
    void launch_update(const DevModel<T>& m, const StepParams<T>& p, int engine, int parity, cudaStream_t st); \
    template <class T>                                                                                         \
    void launch_initdt(const DevModel<T>& m, const StepParams<T>& p, int cur, unsigned long long* out,         \
                       cudaStream_t st);                                                                       \
    template <class T> void launch_volume(const DevModel<T>& m, T delta0, int cur, double* out, cudaStream_t st);
namespace exact {
BGF_DECLARE_LAUNCHERS
}
namespace fast {
BGF_DECLARE_LAUNCHERS
}

// Records the text returned by bgf_last_error() for this thread.
void set_last_error(const std::string& msg);

// Host restatement of the bed preparation the reference performs once at
// initialisation (src/InitialConditions.cu:140-144): bed halo fill and bed
// gradients including halo cells, on BUQ tiles.
template <class T>
int host_bed_gradients(int nblk, const int* active, const int* level, const int* nbr8soa, int nblkmem, double delta,
                       double theta, const T* zb, T* dzbdx, T* dzbdy);

}  // namespace bgf
