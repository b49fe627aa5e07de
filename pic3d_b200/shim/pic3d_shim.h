/* Extra entry points of the C++ drop-in shim (pic3d_shim.cpp) for host code
 * that edits or reads the reference's global arrays outside the calls the
 * shim already keeps coherent.  Include after the reference's particle.h. */
#ifndef PIC3D_SHIM_H
#define PIC3D_SHIM_H

#include <vector>

struct particle;
struct pic_ctx;

/* The GPU context created by initialize_domain (null before it). */
pic_ctx *pic3d_shim_context();

/* Copy the host arrays (ex..bz, jx..jz, rho_particle[0..1]) to the device,
 * and the particle vectors when `particles` is given: for host code that
 * changed them after the shim's first device call. */
void pic3d_shim_push_host(const std::vector<std::vector<particle>> *particles, const int *num_particles);

/* Bring the host arrays, and the particle vectors and counts when given, up
 * to date with the device (needed only with PIC3D_SHIM_LAZY=1). */
void pic3d_shim_pull_host(std::vector<std::vector<particle>> *particles, int *num_particles);

#endif
