/*
 * gen_module.cu — the window kernel's generated-mechanism variants as a module compiled at
 * run time, for mechanisms emitted from MOD files after the library was built
 * (mind_b200.mechanisms.register_mod; loaded by mind_load_mechanisms).
 *
 *     nvcc -cubin -gencode arch=compute_100a,code=sm_100a -DMIND_RUNTIME_MECHANISMS \
 *          -I <dir of runtime_mechanisms.cuh> -I mind.jl_b200/csrc ... gen_module.cu
 *
 * With MIND_RUNTIME_MECHANISMS the device code takes its generated dispatch from
 * runtime_mechanisms.cuh (the compiled-in mechanisms, then the new ones); the entry points
 * below are the library's own window kernel and generated INITIAL, under C names the
 * library looks up in the module.  Not part of libmindgpu.so.
 */
#include "kernels.cuh"

extern "C" {

__global__ void __launch_bounds__(mind::kCellThreads, mind::default_min_blocks(mind::kCellThreads))
    mind_rt_window_fp64(const mind::Params P, const int32_t *cells, int64_t n0, int32_t W) {
    mind::window_body<false, mind::kCellThreads, false, true>(P, cells, n0, W);
}

__global__ void __launch_bounds__(mind::kCellThreads, mind::default_min_blocks(mind::kCellThreads))
    mind_rt_window_mixed(const mind::Params P, const int32_t *cells, int64_t n0, int32_t W) {
    mind::window_body<true, mind::kCellThreads, false, true>(P, cells, n0, W);
}

__global__ void __launch_bounds__(mind::kCellThreads, mind::default_min_blocks(mind::kCellThreads))
    mind_rt_window_fp64_hbm(const mind::Params P, const int32_t *cells, int64_t n0, int32_t W) {
    mind::window_body<false, mind::kCellThreads, true, true>(P, cells, n0, W);
}

__global__ void __launch_bounds__(mind::kCellThreads, mind::default_min_blocks(mind::kCellThreads))
    mind_rt_window_mixed_hbm(const mind::Params P, const int32_t *cells, int64_t n0, int32_t W) {
    mind::window_body<true, mind::kCellThreads, true, true>(P, cells, n0, W);
}

__global__ void mind_rt_generated_init(const mind::Params P, int32_t g) { mind::generated_init_rows(P, g); }

}  // extern "C"
