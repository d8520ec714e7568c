# lj_gpu.pxd -- Cython declarations of the engine's C ABI (lj_gpu.h) for the
# reference's Cython layer (src/python/lennardjonesium/simulation/*.pxd): a
# maintainer copies this file beside _simulation.pxd and cimports it.  The
# struct fields follow lj_gpu.h in order and type.
cdef extern from "lj_gpu.h":
    ctypedef struct lj_params:
        int particle_count
        double box[3]
        double cutoff_distance
        double time_delta
        int precision
        int force_kind
        double force_strength
        int periodic
        int device
        double skin
        int neighbor_capacity
        int force_block
        int mixed_per_pair
    ctypedef struct lj_thermo:
        double time
        double kinetic_energy
        double potential_energy
        double total_energy
        double virial
        double temperature
        double mean_square_displacement
    ctypedef struct lj_ctx
    void lj_gpu_default_params(lj_params*)
    int lj_gpu_create(const lj_params*, lj_ctx**)
    int lj_gpu_destroy(lj_ctx*)
    const char* lj_gpu_last_error(const lj_ctx*)
    int lj_gpu_upload_state(lj_ctx*, const double*, const double*, const double*, const double*, int, double, double, double)
    int lj_gpu_download_state(lj_ctx*, double*, double*, double*, double*, int, double*, double*, double*)
    int lj_gpu_step(lj_ctx*, int, lj_thermo*) nogil
    int lj_gpu_compute_forces(lj_ctx*, double*, double*) nogil
    int lj_gpu_measure(lj_ctx*, lj_thermo*)
    int lj_gpu_set_temperature(lj_ctx*, double, double*)
    int lj_gpu_scale_velocities(lj_ctx*, double)
