// Byte layout of the reference's `struct PT` (include/core/common.h:57-90 of
// MMullerdR/simulador_quantico) with an untyped matrix pointer, so one
// definition serves both amplitude types.  Must stay layout-identical to
// hgm_ref_pt in include/hgm_dropin.h.
#pragma once

struct RefPTLayout {
    int qubits;
    void *matrix;
    int matrix_size;
    int span_start_bit, target_bit;
    bool affected;
    long control_value, control_mask;
    long *control_bit_positions, control_count;
    long *control_rest, control_rest_count;
};

static_assert(sizeof(RefPTLayout) == 80, "struct PT layout (LP64) is 80 bytes");
static_assert(__builtin_offsetof(RefPTLayout, target_bit) == 24, "PT::target_bit offset");
static_assert(__builtin_offsetof(RefPTLayout, control_value) == 32, "PT::control_value offset");
static_assert(__builtin_offsetof(RefPTLayout, control_mask) == 40, "PT::control_mask offset");
