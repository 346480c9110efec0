/*
 * scphd_io.h — file input/output around the filter step: the configuration file,
 * measurement sequences and result files of the reference's driver.
 *
 *   reference                                          this ABI
 *   libconfig read in the constructor (.cu:827-1005,   scphd_config_from_file
 *     1145, 1343, 1744, 1920, 2596-2610, 2655) and in
 *     main (src/main.cpp:72-77)
 *   readMatfile(filename, "Z1"/"Z2") (src/main.cpp:19-50) scphd_read_mat_frames
 *   writeMat(filename) (src/scphdcameracalibration.cu:2200-2373, matio)
 *                                                      scphd_write_mat
 *
 * Files are MATLAB level-5 MAT files (the reference's fixtures are level 5 with zlib
 * compression; the reference writes level 7.3, which MATLAB loads the same way).
 * The host-only parts (configuration, reading, scphd_write_mat_arrays) need no GPU.
 */
#ifndef SCPHD_IO_H
#define SCPHD_IO_H

#include "scphd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Driver settings that the reference reads outside the filter (src/main.cpp:72-77,
 * writeMat's save_all_maps). */
typedef struct scphd_run_options {
    int32_t max_steps;       /* max_steps (default: all frames) */
    int32_t slam;            /* slam: every frame from camera 2, not fixed (default 0) */
    int32_t save_all_maps;   /* save_all_maps: also write the per-parent mixtures (default 0) */
    int32_t verbosity;       /* verbosity (default 0) */
} scphd_run_options;

/* Read a configuration file in the reference's libconfig syntax (settings "name =
 * value" or "name : value", ';' or ',' optional, groups { }, '#', '//' and block
 * comments) onto cfg and opts, which hold their defaults on entry (scphd_config_defaults).
 * Keys the reference's code reads: n_particles, particles_per_feature, min_weight,
 * min_separation, min_neff, ps, prior.{cartesian,angular}.{x,y,z,vx,vy,vz}.{a,b} (a
 * uniform box; the shipped file's {mean,std} is accepted as mean -/+ std),
 * camera_motion_model.{cartesian,angular}.{ax,ay,az}, feature_motion_model.{ax,ay,az},
 * measurement_model.{fx,fy,u0,v0,std_u,std_v,pd,lambda} (kappa = lambda / (2 v0)^2,
 * src/disparitymeasurementmodel.cu:157-162), birth.{w0,d0,vu0,vv0,vd0,var_d0,var_vu0,
 * var_vv0,var_vd0}, max_steps, slam, save_all_maps, verbosity.  Keys of this
 * implementation, optional: max_gaussians, max_measurements, max_survivors, meas_dim,
 * precision ("fp32"/"fp64" or 0/1), seed, device, baseline, measurement_model.std_d.
 * Unknown keys are ignored (the reference ignores max_velocity and min_range on this
 * path).  Errors name the file, line and key. */
scphd_status scphd_config_from_file(const char* path, scphd_config* cfg, scphd_run_options* opts);

/* Read variable `var` of a MAT file: a cell array of K frames, each a 2 x n (u; v) or
 * 3 x n (u; v; d) real matrix (other numeric storage types are converted).  First call
 * with sizes == NULL and data == NULL to get *n_frames and *rows; then with sizes
 * holding n_frames entries and data holding rows * sum(sizes) values, frame after frame,
 * each frame row-major (all u, then all v, then all d). */
scphd_status scphd_read_mat_frames(const char* path, const char* var, int32_t* n_frames, int32_t* rows,
                                   int32_t* sizes, double* data, int64_t data_capacity);

/* Write the filter's state as writeMat does: "particles" (12 x N), "weights" (N x 1,
 * normalised linear), "log_weights" (N x 1, an addition), and the struct "features"
 * with the MAP parent's map: "weights" (n x 1) and "particles" (6 x n*P world samples,
 * feature after feature).  With save_all_maps, also the per-parent mixtures of the last
 * update as N x 1 struct arrays {weights 1 x n, means 6 x n, covs 6 x 6 x n}:
 * "features_predicted" (the refitted prediction) and "features_merged"; the reference's
 * "features_updated" (every Gaussian x measurement pair) is never materialised here
 * and is written empty. */
scphd_status scphd_write_mat(scphd_filter* f, const char* path, int32_t save_all_maps);

/* Write named real matrices (column-major, as MATLAB stores them) to a MAT file. */
scphd_status scphd_write_mat_arrays(const char* path, int32_t n, const char* const* names, const int32_t* rows,
                                    const int32_t* cols, const double* const* data);

#ifdef __cplusplus
}
#endif

#endif
