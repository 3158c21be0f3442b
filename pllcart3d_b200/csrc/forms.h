// Entry points of the two precision forms (form_f64.cu, form_f32.cu).
#pragma once

struct pllgpu_ctx;

namespace pll {

void form_enqueue_step_f64(pllgpu_ctx* c);
void form_enqueue_step_f32(pllgpu_ctx* c);
int form_start_f64(pllgpu_ctx* c);
int form_start_f32(pllgpu_ctx* c);
int form_resume_f64(pllgpu_ctx* c);
int form_resume_f32(pllgpu_ctx* c);
int form_routine_f64(pllgpu_ctx* c, int routine, const double* in, double* out);
int form_routine_f32(pllgpu_ctx* c, int routine, const double* in, double* out);
int form_materialize_f64(pllgpu_ctx* c);
int form_materialize_f32(pllgpu_ctx* c);
void* form_field_ptr_f64(pllgpu_ctx* c, int f);
void* form_field_ptr_f32(pllgpu_ctx* c, int f);
void form_diag_f64(pllgpu_ctx* c);
void form_diag_f32(pllgpu_ctx* c);
bool form_alloc_f64(pllgpu_ctx* c);
bool form_alloc_f32(pllgpu_ctx* c);
// the FP64 form with FP32 WENO5 weights (form_f64m.cu)
void form_enqueue_step_f64m(pllgpu_ctx* c);
int form_start_f64m(pllgpu_ctx* c);
int form_resume_f64m(pllgpu_ctx* c);
int form_routine_f64m(pllgpu_ctx* c, int routine, const double* in, double* out);
int form_materialize_f64m(pllgpu_ctx* c);
void* form_field_ptr_f64m(pllgpu_ctx* c, int f);
void form_diag_f64m(pllgpu_ctx* c);
bool form_alloc_f64m(pllgpu_ctx* c);
// the exact FP64 form (form_f64x.cu)
void form_enqueue_step_f64x(pllgpu_ctx* c);
int form_start_f64x(pllgpu_ctx* c);
int form_resume_f64x(pllgpu_ctx* c);
int form_routine_f64x(pllgpu_ctx* c, int routine, const double* in, double* out);
int form_materialize_f64x(pllgpu_ctx* c);
void* form_field_ptr_f64x(pllgpu_ctx* c, int f);
void form_diag_f64x(pllgpu_ctx* c);
bool form_alloc_f64x(pllgpu_ctx* c);

// runtime.cu: the field of id f in the form's storage type, with the
// reference's new == old view after fast steps (a write materialises "new")
void* field_ptr(pllgpu_ctx* c, int f, bool for_write);
// one full step of either form on the context's stream (runtime.cu)
void enqueue_step_any(pllgpu_ctx* c);
int materialize(pllgpu_ctx* c);

}  // namespace pll
