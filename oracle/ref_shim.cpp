// ref_shim.cpp -- test infrastructure only.  Gives the reference's own CPU
// propagator (compiled unmodified from TorchWI's sources by oracle/Makefile)
// plain C entry points so the tests can call it through ctypes.  The
// wrapped functions are declared in torchwi/propagator/td2d/propagator_cpu.h
// (c_fdm_forward / c_fdm_backward) and defined in propagator_cpu.cpp:5-152
// and propagator_forward_cpu.cpp:5-71 of the reference.
#include "propagator_cpu.h"

extern "C" {

void ref_fdm_forward(float* frd, float* virt, float* u1, float* u2, float* u3,
                     float* vel, float* w, int order, int dimx, int dimy, int nt,
                     float h, float dt, float sx, float sy, float ry) {
    c_fdm_forward(frd, virt, u1, u2, u3, vel, w, order, dimx, dimy, nt, h, dt,
                  sx, sy, ry);
}

void ref_fdm_backward(float* grad, float* virt, float* u1, float* u2, float* u3,
                      float* vel, float* resid, int order, int dimx, int dimy,
                      int nt, float h, float dt, float ry) {
    c_fdm_backward(grad, virt, u1, u2, u3, vel, resid, order, dimx, dimy, nt, h,
                   dt, ry);
}

void ref_fdm_forward_only(float* frd, float* u1, float* u2, float* u3,
                          float* vel, float* w, int order, int dimx, int dimy,
                          int nt, float h, float dt, float sx, float sy,
                          float ry) {
    c_fdm_forward_only(frd, u1, u2, u3, vel, w, order, dimx, dimy, nt, h, dt,
                       sx, sy, ry);
}

}  // extern "C"
