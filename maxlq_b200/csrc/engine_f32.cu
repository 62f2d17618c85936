// engine_f32.cu -- Engine<float>: the mixed-precision (FP32 fields) pipelines.
#include "engine_impl.cuh"

namespace mlq {
template class Engine<float>;
}  // namespace mlq
