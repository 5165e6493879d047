// serve.cu -- the serving launch (serve_kernel and its launchers, declared in
// engine.hpp), compiled as a translation unit of its own from the decoder's
// source. Its overflow decoders run the decoder body on a tile in global
// memory; compiled beside the batch kernels, that gives the out-of-line
// helpers they share (seeding, FSR) generic pointers, and the batch decoder
// loses its shared-memory addressing: 184 instead of 168 registers and a
// slower batched step. Apart, each translation unit keeps its own copies.
#define PLP_SERVE_TU
#include "decoder.cu"
