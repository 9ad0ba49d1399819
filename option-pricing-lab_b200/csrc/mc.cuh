// Fused pricing plan: a checked ob_mc_request packed for the device, launched any number of times.
#pragma once

#include "fused.cuh"

namespace ob {

// Byte offsets of each array inside the packed blob (16-byte aligned).
struct McOffsets {
    int dt, root, kind, cvar, hes, step_row, lo, inv_dx, lf, obs_of_step, ln_trig, obs_disc, leg_type, leg_strike,
        leg_barrier, ln_level, table, t0, low_root;
};

template <typename R>
struct McArgs {
    McOffsets off;
    const unsigned char* blob;  // device copy of the blob, staged into shared memory by each block
    int smem_blob;              // bytes of the blob copied to shared memory (table included when it fits)
    int table_in_smem;
    const R* table_global;      // the table, when it stays in global memory
    int n_names, n_steps, n_x, same, has_var, has_slv;
    int mixer;   // local correlation: t0 and low_root staged, mix the constants
    R mix[8];
    int n_out, n_legs, n_obs;
    QeConsts<R> qe;
    R spot0;
    double discount;
    // autocall
    int has_coupon, memory, ki_daily;
    R ln_cb, ln_ki;
    double coupon, put_strike;
};

void check_mc_request(const ob_mc_request& rq);
void check_mc_model(const ob_mc_request& rq);  // the model part of an ob_mc_request (its product unused)

struct McPlan {
    DeviceArena arena;
    int precision = OB_FP32;
    int n_out = 0, sms = 0, blocks_per_sm = 1, max_blocks = 0;
    int block = 256, grid_waves = 1;
    int threads_per_pair = 1;  // 2: the QE kernel runs the two legs of a pair on two lanes
    bool force_generic = false;  // tests: run the generic kernel even where the specialised one applies
    size_t smem_bytes = 0;
    const void* kernel = nullptr;
    McArgs<float> args_f{};
    McArgs<double> args_d{};
    double* d_partial = nullptr;
    double* d_sums = nullptr;
    long long pairs_run = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    bool timing = false;
    cudaStream_t last_stream = nullptr;
    bool fused = false;  // the specialised kernel of fused.cu runs this plan
    FusedArgs<float> fa_f{};
    FusedArgs<double> fa_d{};

    template <typename R>
    FusedArgs<R>& fused_args();

    template <typename R>
    McArgs<R>& args();
    template <typename R>
    void build(const ob_mc_request& rq);
    void create(const ob_mc_request& rq, int precision);
    int launch_shape(long long n_pairs, int& blk);
    int occupancy_at(int blk);
    int occ_block[16] = {}, occ_blocks[16] = {};  // resident blocks a SM at other block sizes, as queried
    void run(long long n_pairs, long long first_pair, unsigned long long seed, cudaStream_t st);
    void result(ob_mc_result& res);
    ~McPlan();
};

template <>
inline FusedArgs<float>& McPlan::fused_args<float>() {
    return fa_f;
}
template <>
inline FusedArgs<double>& McPlan::fused_args<double>() {
    return fa_d;
}

template <typename R>
bool fused_build(McPlan& plan, const ob_mc_request& rq);

template <>
inline McArgs<float>& McPlan::args<float>() {
    return args_f;
}
template <>
inline McArgs<double>& McPlan::args<double>() {
    return args_d;
}

}  // namespace ob
