/*
 * hgm_dropin.h -- the reference's GPU-backend C-ABI, as exported by
 * libhgm_dropin_f32.so / libhgm_dropin_f64.so.
 *
 * These are exactly the four symbols the reference's DGM engine binds for its
 * GPU backend (declared at include/core/dgm.h:23,30-32 of
 * MMullerdR/simulador_quantico, defined at src/core/kernel.cu:31,303,321,384,
 * stub shape at src/core/kernel_stub.cpp:15-33).  Linking either library in
 * place of the reference's kernel.o (makefile:51-61) runs the reference's
 * general.out / grover.out unchanged on this engine.
 *
 * Two builds, one per amplitude type:
 *   libhgm_dropin_f32.so  `complex float`  -- the unmodified reference
 *   libhgm_dropin_f64.so  `complex double` -- the FP64-widened reference
 * Define HGM_DROPIN_F64 before including this header to get the FP64
 * prototypes.
 *
 * Error behaviour follows the reference: a CUDA or planning failure prints a
 * message and calls exit(1) (src/core/kernel.cu:439-447); setDevice returns
 * the CUDA error as a bool (false on success, src/core/kernel.cu:31-33).
 */
#ifndef HGM_DROPIN_H
#define HGM_DROPIN_H

#include <stdbool.h>

#ifdef __cplusplus
typedef float __complex__ hgm_cfloat;
typedef double __complex__ hgm_cdouble;
extern "C" {
#else
typedef float _Complex hgm_cfloat;
typedef double _Complex hgm_cdouble;
#endif

#ifdef HGM_DROPIN_F64
typedef hgm_cdouble hgm_dropin_amp;
#else
typedef hgm_cfloat hgm_dropin_amp;
#endif

/*
 * Memory layout of the reference's `struct PT` (include/core/common.h:57-90):
 * a compiled controlled 1-qubit gate.  Only target_bit, control_mask,
 * control_value and matrix are read; the remaining fields are kept so the
 * layout (80 bytes on LP64) matches the reference objects.
 */
typedef struct hgm_ref_pt {
    int qubits;
    hgm_dropin_amp *matrix;       /* row-major [m00, m01, m10, m11] */
    int matrix_size;
    int span_start_bit, target_bit;
    bool affected;
    long control_value, control_mask;
    long *control_bit_positions, control_count;
    long *control_rest, control_rest_count;
} hgm_ref_pt;

/* src/core/kernel.cu:31-33 -- CUDA context warm-up on device `device_id`.
 * Returns the CUDA error as a bool (false on success). */
bool setDevice(int device_id);

/* src/core/kernel.cu:303-316 -- applies the NULL-terminated PT list `pts`
 * `iterations` times to the host state `read_memory` (2^qubits amplitudes,
 * updated in place, same pointer returned).  coalesced_bits,
 * gpu_region_bits, block_size and repeat_count are validated with the
 * reference's rules (2*block_size*repeat_count == 2^gpu_region_bits,
 * gpu_region_bits >= coalesced_bits, dgm_core.cpp:207-223); the engine then
 * chooses its own tiles.  gpu_count > 1 runs on one GPU with a notice on
 * stderr (the multi-GPU peer mode is not provided). */
hgm_dropin_amp *GpuExecutionWrapper(hgm_dropin_amp *read_memory, hgm_ref_pt **pts, int qubits,
                                    int coalesced_bits, int gpu_region_bits, int gpu_count,
                                    int block_size, int repeat_count, int iterations);

/* src/core/kernel.cu:321-380 and :384-435 -- the hybrid CPU+GPU mode's
 * region projection.  The hybrid mode is not provided: both print a notice
 * and return false, as src/core/kernel_stub.cpp:25-33 does. */
bool ProjectState(hgm_dropin_amp *state, int qubits, int region_size, long region_id, long region_mask,
                  int gpu_count);
bool GetState(hgm_dropin_amp *state, int qubits, int region_size, long region_id, long region_mask,
              int gpu_count);

#ifdef __cplusplus
}
#endif
#endif /* HGM_DROPIN_H */
