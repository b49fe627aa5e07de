// Launchers shared between the translation units of libpic3d_b200.so.
#pragma once

#include "pic_internal.cuh"

namespace pic {

// profiling: CUDA events around each launch when pic_profile_enable(1)
void prof_begin(pic_ctx *c, const char *name);
void prof_end(pic_ctx *c);

// field_kernels.cu
void launch_update_e(pic_ctx *c, double coef);   // E += coef (curl B - J), then the E ghost fill
void launch_update_b(pic_ctx *c, double coef);   // B -= coef curl E, then the B ghost fill
void launch_ghost_fill_one(pic_ctx *c, int array);
void launch_fold_currents(pic_ctx *c, unsigned mask = 31u);
void launch_radiating_boundary(pic_ctx *c, int is_left, int is_right, int step);
void launch_absorbing_faces(pic_ctx *c);   // PicParams.absorbing extension (with the radiating boundary)
void launch_binomial_pass(pic_ctx *c, int ring_index, int axis, void *scratch);
int launch_eval(pic_ctx *c, int what, const double *in, double *d_out);

// particle_kernels.cu
// device generators of reference records (staging buffer `rec`, records
// [off, off + n) of the species)
struct LatticeArgs {
    void *rec;
    long long n, off;
    const double *ax, *ay, *az;   // coordinates of the kept lattice indices per axis
    const double *wx;             // weight per kept x index, or null: wconst
    double wconst;
    long long nvx, nvy;
    double p[3], s[3], gamma, charge, mass;
};
struct ThermalArgs {
    void *rec;
    long long n, off;
    int nx, ny, ppc;
    unsigned key0, key1;
    double u_th, weight, charge, mass;
};
void launch_lattice_records(pic_ctx *c, const LatticeArgs &a);
void launch_thermal_records(pic_ctx *c, const ThermalArgs &a);
void launch_push(pic_ctx *c, int kind);
// idx: (index, home tile) pairs; visitors recorded into v when v.raw is set
void launch_push_list(pic_ctx *c, int kind, const int *idx, const unsigned long long *count, const VisSink &v);
void launch_remove(pic_ctx *c, int kind);
void launch_upload_particles(pic_ctx *c, int kind, const void *d_records, int64_t n, int64_t offset,
                             unsigned long long *check = nullptr);
void launch_download_particles(pic_ctx *c, int kind, void *d_records, int64_t n, int64_t offset);
void launch_convert_array(pic_ctx *c, void *dst, const void *src, long long n, int to_device);
void launch_iota(pic_ctx *c, int *a, long long n);   // a[i] = i
void launch_deposit_one(pic_ctx *c, int kind, const double (&xo)[3], const double (&xn)[3], double qw);

// tile_kernels.cu
void launch_sort(pic_ctx *c, int kind);
void launch_sort_due(pic_ctx *c, int mask);   // the sorts the next push of the masked species needs
void launch_tile_push(pic_ctx *c, int mask);
int tile_order_stats(pic_ctx *c, int kind, long long (&out)[4]);
VisSink vis_sink_of(const pic_ctx *c, const Species &s);   // where a push of species s records visitors
// Row and plane strides of a tile kernel's shared box of extent e for tile
// edge T (padded so that 32 consecutive cells of a tile start in different
// banks).
__host__ __device__ constexpr int padded_row(int e, int T) {
    int sy = e;
    while (sy % (2 * T) != T) ++sy;
    return sy;
}
__host__ __device__ constexpr int padded_plane(int e, int T) {
    int sz = e * padded_row(e, T);
    while (sz % (2 * T * T) != (T * T) % (2 * T * T)) ++sz;
    return sz;
}

// the tile kernels' shared boxes: gather box of GE points per axis (row and
// plane strides gsy, gsz, gsize elements), deposit box of DE (dsy, dsz, dsize)
struct TileBoxes {
    int GE, DE, gsy, gsz, gsize, dsy, dsz, dsize;
};
TileBoxes tile_boxes(const pic_ctx *c);
size_t tile_smem_bytes(const pic_ctx *c);

// adjoint_kernels.cu
void adjoint_record_hook(pic_ctx *c);

// diag_kernels.cu
void launch_diagnostics(pic_ctx *c, double *d_out);

}  // namespace pic
