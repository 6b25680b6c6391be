// hg_engine_fp32.cu -- the chosen form: Engine<float> (FP32 mesh, transforms and fields;
// FP64 sums, scalars and shot-noise histograms; optional FP64 stages).
#define HG_TU_NS tu_fp32
#include "hg_engine.cuh"

namespace hg {
hg_ctx *make_engine_fp32(const hg_config &c) { return new Engine<float>(c); }
}  // namespace hg
