// hg_engine_fp64.cu -- the plain form: Engine<double> (FP64 throughout, as the reference).
#define HG_TU_NS tu_fp64
#include "hg_engine.cuh"

namespace hg {
hg_ctx *make_engine_fp64(const hg_config &c) { return new Engine<double>(c); }
}  // namespace hg
