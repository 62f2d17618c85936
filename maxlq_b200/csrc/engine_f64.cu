// engine_f64.cu -- Engine<double>: the all-FP64 pipelines.
#include "engine_impl.cuh"

namespace mlq {
template class Engine<double>;
}  // namespace mlq
