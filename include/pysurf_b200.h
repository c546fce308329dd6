/*
 * pysurf_b200.h -- C-ABI of the B200 delta-SPH backend (libpysurf_b200.so).
 *
 * The drop-in boundary is the solver-backend interface pySurf's WcsphSolver drives,
 * `pysurf.sphGpu.PairSums` (src/pysurf/sphGpu.py:1482-2323).  Each entry point below replaces one
 * method of it; the citation on each names the method.  A Python `PairSums` over this ABI lives in
 * pysurf_b200/sphGpu.py; a ctypes or cffi binding needs nothing but these declarations.
 *
 * Conventions
 *   - Plain pointers and sizes only.  Unless a name ends in _device, array arguments are HOST
 *     memory, row-major float64 as numpy lays them out: vectors (n, dim), matrices (n, dim, dim),
 *     scalars (n,); fluid flags one byte per particle.  The library copies inputs in and results
 *     out through its own pinned staging; the caller keeps ownership of every array it passes.
 *   - Every call returns 0 (SPH_OK) or a negative status; sph_last_error() describes the last
 *     failure on the calling thread.
 *   - A handle is one particle system on one device; calls on one handle must not overlap.
 *     Work is ordered on the handle's stream (sph_set_stream; the device's default stream
 *     otherwise).  Calls that return host results synchronize that stream.
 *   - The library allocates its own device memory (float64 master state, float32 sweep frame,
 *     sort scratch), about 300 bytes a particle in 2D, and frees it in sph_destroy.
 */
#ifndef PYSURF_B200_H
#define PYSURF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPH_OK 0
#define SPH_ERR_INVALID (-1)     /* an argument is out of range; no state changed */
#define SPH_ERR_NOMEM (-2)       /* device or pinned host memory ran out */
#define SPH_ERR_CUDA (-3)        /* a CUDA call failed */
#define SPH_ERR_NONFINITE (-4)   /* the state stopped being finite during a step */
#define SPH_ERR_TIMESTEP (-5)    /* the time step collapsed (not positive and finite) */
#define SPH_ERR_STATE (-6)       /* the call needs state the handle does not hold yet */
#define SPH_ERR_CAPACITY (-7)    /* an output array is too small; the needed size is returned */
#define SPH_ERR_UNSUPPORTED (-8) /* an option the backend does not carry */

typedef struct SphSystem SphSystem;

/* Construction: PairSums.__init__ (src/pysurf/sphGpu.py:1524-1569).
 * kernel_type 0 cubic spline, 1 Wendland C2; period > 0 makes y periodic (3D only);
 * precise 1 takes separations from the float64 positions' point and remainder, 0 from the
 * float32 points alone (separationPrecision). */
int sph_create(int dimensions, double smoothing_length, const double *domain_min, const double *domain_max,
               double period, int precise, int kernel_type, int device, SphSystem **out);
int sph_destroy(SphSystem *sys);
const char *sph_last_error(void);
int sph_version(void);
/* The architecture the library's kernels were compiled for, as the CUDA runtime loads them on the
 * current device (cudaFuncAttributes.binaryVersion: 100 for sm_100a).  No counterpart in the
 * reference: a diagnostic that the loaded library carries B200 code. */
int sph_kernel_architecture(int *version);

/* The hash grid's shape the reference's sortParticles reads (PairSums.gridShape,
 * src/pysurf/sphGpu.py:1466-1478 gridDimensions). */
int sph_grid_shape(const SphSystem *sys, int64_t shape[3]);
/* Cells per support of the internal cell list (1: cells 2h wide, 2: cells h wide, ...; the
 * default 3, cells 2h / 3 wide, offers the fewest candidates for the stencil's cost). */
int sph_set_cells_per_support(SphSystem *sys, int cells);
/* How the sweeps find neighbours: neighbor_table 1 (the default) records each step's neighbours
 * once, after the cell list, in a table sized to the largest count seen at push/update plus a
 * quarter, when it fits in three quarters of the free device memory; a particle whose count
 * outgrows its row walks the cells, with the same summation order.  0 always walks the cells.
 * threads_per_particle 1, 2, 4 (the default) or 8 threads share each particle's neighbours (sums
 * combined by shuffles in a fixed order). */
int sph_set_sweep_options(SphSystem *sys, int neighbor_table, int threads_per_particle);
/* The neighbour table's row capacity now (0: the sweeps walk the cells). */
int sph_neighbor_table(const SphSystem *sys, int64_t *row_capacity);
/* The CUDA stream (a cudaStream_t) the handle's work goes on; NULL for the default stream. */
int sph_set_stream(SphSystem *sys, void *stream);

/* Setters: PairSums.setDiffusion (src/pysurf/sphGpu.py:1882), setWallPressure (1910),
 * setNegativePressure (1921), setContinuityCorrection (1701), setViscosityLimiter (1744).
 * mode 0 none, 1 molteni, 2 hydrostatic, 3 antuono. */
int sph_set_diffusion(SphSystem *sys, int mode, double delta, double sound_speed, double reference_density,
                      double gravity);
int sph_set_wall_pressure(SphSystem *sys, int extrapolated);
int sph_set_negative_pressure(SphSystem *sys, int enabled);
int sph_set_continuity_correction(SphSystem *sys, int enabled);
int sph_set_viscosity_limiter(SphSystem *sys, int enabled);
/* PairSums.setClosure (src/pysurf/sphGpu.py:1752-1779): the delta-LES-SPH closure on or off, with
 * c0, rho0 and the water's kinematic viscosity.  When on, every step takes each particle's alpha_i
 * and delta_i from its velocity gradient (src/pysurf/sphSolver.py:1232-1274), adds the closure's
 * viscous term to every fluid pair's accelerations and takes each fluid pair's diffusion
 * coefficient as the harmonic mean of the two deltas. */
int sph_set_closure(SphSystem *sys, int enabled, double sound_speed, double reference_density,
                    double kinematic_viscosity);
/* PairSums.setShifting (src/pysurf/sphGpu.py:1927-1957): particle shifting on or off, with the
 * Mach number of its size CFL Ma (2h)^2, the particle spacing (for the anti-clumping weight's
 * W(dx)), c0, and whether each particle's size is 2 h |v_i| dt instead (local).  It needs one
 * smoothing length for every particle.  When on, each device step shifts the fluid after the
 * density update, from the step's starting geometry (src/pysurf/sphSolver.py:1760-1785). */
int sph_set_shifting(SphSystem *sys, int enabled, double mach, double spacing, double sound_speed, int local);
/* PairSums.shiftingDisplacement (src/pysurf/sphGpu.py:1980-1995): this step's shift (n, dim), density
 * change (n) and velocity change (n, dim) of every particle, caller order, zero on the boundary and
 * the free surface. */
int sph_shifting_displacement(SphSystem *sys, const double *densities, double time_step, const double *velocities,
                              double *shifts, double *density_changes, double *velocity_changes);
/* PairSums.setEnergyBudget (src/pysurf/sphGpu.py:1780-1792): whether the device steps keep the energy
 * budget (src/pysurf/sphEnergy.py): each fluid particle's running total of every term from the last
 * sph_push, 120 bytes a particle more while it is on. */
int sph_set_energy_budget(SphSystem *sys, int enabled);
/* Compensated momentum and continuity sums (no method of PairSums: the reference's float32 Warp
 * sums are plain, src/pysurf/sphGpu.py:400-414, 476-545; its float64 numpy path is the accuracy they
 * approach).  When on, each thread's share of a particle's du/dt and drho/dt is accumulated with its
 * running rounding error (the Dot2 scheme of Ogita, Rump and Oishi, 2005) and the threads' shares
 * combine the same way, so the sums lose no digits to their length; the terms keep their float32
 * arithmetic.  Off by default.  SPH_ERR_UNSUPPORTED with the energy budget on (its sweeps keep
 * plain sums). */
int sph_set_compensated_sums(SphSystem *sys, int enabled);
/* PairSums.energySums (src/pysurf/sphGpu.py:1805-1825): each term's energy [J] over the device steps
 * since sph_push, summed over the particles in caller order, into sums[14], in the order pressureFluid,
 * viscosityFluid, pressureWall, viscosityWall, gravityWork, continuityFluid, continuityWall,
 * correction, diffusion, floor, drift, clamp, shifting, filter.  SPH_ERR_STATE while the budget is off. */
int sph_energy_sums(SphSystem *sys, double *sums);
/* The fluid's kinetic, potential (-m g . x) and elastic energy [J] of the device state into
 * energies[3] (src/pysurf/sphParticles.py:236-255, src/pysurf/sphSolver.py:2156-2161): the budget's
 * terms sum to the change of their total, and a split's change of it is the refinement term. */
int sph_fluid_energy(SphSystem *sys, double *energies);
/* PairSums.closureCoefficients (src/pysurf/sphGpu.py:1841-1853): alpha_i and delta_i, caller order. */
int sph_closure_coefficients(SphSystem *sys, const double *velocities, const double *densities, double *alphas,
                             double *deltas);
/* PairSums.setPhysics (src/pysurf/sphGpu.py:2173-2205); density_floor in kg/m^3, 0 for none. */
int sph_set_physics(SphSystem *sys, double reference_density, double sound_speed, double alpha,
                    double boundary_viscosity_factor, const double *gravity, double xsph_epsilon,
                    double density_floor);

/* ---- Host steps (the state stays with the caller) ---------------------------------------- */

/* PairSums.update (src/pysurf/sphGpu.py:1998-2042): positions, masses, flags and lengths
 * (lengths may be NULL for the handle's h throughout); rebuilds the cell list.  Fails with
 * SPH_ERR_INVALID when a length exceeds the handle's h. */
int sph_update(SphSystem *sys, int64_t n, const double *positions, const double *masses, const uint8_t *is_fluid,
               const double *lengths);
/* PairSums.pairAccelerations (src/pysurf/sphGpu.py:2044-2059) -> out (n, dim). */
int sph_pair_accelerations(SphSystem *sys, const double *velocities, const double *densities,
                           const double *pressures, double sound_speed, double alpha, double boundary_factor,
                           const double *gravity, double *out);
/* PairSums.continuityRate (src/pysurf/sphGpu.py:2061-2078) -> out (n,); densities may be NULL
 * only without diffusion and correction. */
int sph_continuity_rate(SphSystem *sys, const double *velocities, const double *densities, double *out);
/* PairSums.xsphVelocity (src/pysurf/sphGpu.py:2080-2088) -> out (n, dim). */
int sph_xsph_velocity(SphSystem *sys, const double *velocities, const double *densities, double epsilon,
                      double *out);
/* PairSums.wallPressure (src/pysurf/sphGpu.py:2090-2102) -> out (n,), the boundary's replaced. */
int sph_wall_pressure(SphSystem *sys, const double *densities, const double *pressures, const double *gravity,
                      double reference_density, double sound_speed, double *out);
/* PairSums.shepardDensity (src/pysurf/sphGpu.py:2104-2113) -> out (n,). */
int sph_shepard_density(SphSystem *sys, const double *densities, double *out);
/* PairSums.velocityGradients (src/pysurf/sphGpu.py:1827), correctionMatrices (1855),
 * densityGradients (1868) -> (n, dim, dim), (n, dim, dim), (n, dim). */
int sph_velocity_gradients(SphSystem *sys, const double *velocities, const double *densities, double *out);
int sph_correction_matrices(SphSystem *sys, const double *densities, double *out);
int sph_density_gradients(SphSystem *sys, const double *densities, double *out);

/* ---- Device-resident steps (the state lives on the device between push and pull) --------- */

/* PairSums.push (src/pysurf/sphGpu.py:2207-2221): the whole state, caller order.  Returns once the
 * host arrays have been read; the device's own work on them follows in stream order. */
int sph_push(SphSystem *sys, int64_t n, const double *positions, const double *velocities, const double *densities,
             const double *masses, const uint8_t *is_fluid, const double *lengths);
/* PairSums.pull (src/pysurf/sphGpu.py:2223-2235): any output may be NULL.  masses, lengths and
 * is_fluid come back too, since a device split changes them.  Pressures are the frame's, the ones
 * the last step used; after a push, split or merge with no step since, they are the Tait pressures
 * of the densities and the accelerations are zero (no step has taken them for that state). */
int sph_pull(SphSystem *sys, double *positions, double *velocities, double *densities, double *pressures,
             double *accelerations, double *masses, double *lengths, uint8_t *is_fluid);
/* sph_push and sph_pull over DEVICE arrays on the handle's device (a torch tensor's data_ptr(),
 * float64 contiguous, the same shapes), copied device to device on the handle's stream, so a
 * caller whose state lives in device tensors never routes it through the host.  The push reads
 * the lengths back to check them on the host (n doubles); both return once their copies are done
 * (the handle's stream is synchronized), so the caller's tensors are free, or hold the results,
 * whatever stream the caller works on.  Same citations as sph_push and sph_pull. */
int sph_push_device(SphSystem *sys, int64_t n, const double *positions, const double *velocities,
                    const double *densities, const double *masses, const uint8_t *is_fluid, const double *lengths);
int sph_pull_device(SphSystem *sys, double *positions, double *velocities, double *densities, double *pressures,
                    double *accelerations, double *masses, double *lengths, uint8_t *is_fluid);
int sph_count(const SphSystem *sys, int64_t *n);
/* FrameWriter.write's arrays from the device state (src/pysurf/sphFrames.py:60-100): every
 * particle's float32 position (n x dim) and float32 speed, the speed |v| taken in float64 as numpy
 * takes it, and its fluid flag, in caller order; the caller keeps the fluid rows.  17 bytes a
 * particle in 3D cross the bus instead of a float64 pull's 48. */
int sph_frame(SphSystem *sys, float *positions, float *speeds, uint8_t *is_fluid);

/* PairSums.setBoundary (src/pysurf/sphGpu.py:2121-2171), one call per kind. */
int sph_clear_boundary(SphSystem *sys);
int sph_set_boundary_container(SphSystem *sys, const double *lower, const double *upper, int open_top);
/* bed: the profile's vertices; clearance = spacing / 4; side walls in 3D at y = clearance and
 * width - clearance; the offshore wall at wall_x with the piston's speed; end_limit the
 * shoreward limit. */
int sph_set_boundary_bed(SphSystem *sys, const double *bed_x, const double *bed_z, int64_t count, double clearance,
                         int side_walls, double width, int offshore_wall, double wall_x, double piston_speed,
                         double end_limit);
/* height field: table (ny, nx) row-major, grid origin and steps, walls as HeightFieldBoundary. */
int sph_set_boundary_height_field(SphSystem *sys, const double *table, int64_t nx, int64_t ny, double origin_x,
                                  double origin_y, double step_x, double step_y, double clearance, double low_y,
                                  double high_y, int offshore_wall, double low_x, double high_x);
/* PairSums.enforceBoundary (src/pysurf/sphGpu.py:2317-2323). */
int sph_enforce_boundary(SphSystem *sys);

/* PairSums.residentRates (src/pysurf/sphGpu.py:2237-2273): the first half of a device step;
 * returns the largest fluid speed and acceleration. */
int sph_resident_rates(SphSystem *sys, int filter_density, double *max_speed, double *max_acceleration);
/* PairSums.residentIntegrate (src/pysurf/sphGpu.py:2275-2315): the second half, with the host's dt. */
int sph_resident_integrate(SphSystem *sys, double time_step);

/* WcsphSolver.advance's device loop (src/pysurf/sphSolver.py:1941-1991) without a host round trip
 * per step: steps while time < until_time and step < max_step, each step's dt taken on the
 * device from its own maxima (cflTimeStep, src/pysurf/sphSolver.py:1410-1424); a Shepard filter
 * step every filter_interval steps (0 for none).  On return *time, *step and *last_dt hold the
 * clock.  Steps are captured once into a CUDA graph and replayed. */
int sph_advance(SphSystem *sys, double *time, int64_t *step, double *last_dt, double until_time, int64_t max_step,
                double shortest_length, double cfl, double max_time_step, int64_t filter_interval);

/* ---- Utilities ----------------------------------------------------------------------------- */

/* cellOrderKey (src/pysurf/sphSolver.py:1379-1408), float64, bit-exact: keys (n,). */
int sph_cell_order_key(const double *positions, int64_t n, int dimensions, double cell_width, const int64_t *shape,
                       int64_t *keys, int device);
/* sphCompiled.neighborList (src/pysurf/sphCompiled.py:133-234) of the handle's current positions
 * (after sph_update or sph_push): every particle's neighbours closer than radius, itself
 * excluded, by the same float64 test, so each row holds the reference's set bit for bit; rows in
 * the walk's order.  offsets has n + 1 entries; when capacity < the total, SPH_ERR_CAPACITY and
 * *total set. */
int sph_neighbor_list(SphSystem *sys, double radius, int64_t *offsets, int32_t *neighbors, int64_t capacity,
                      int64_t *total);
/* splitParticles (src/pysurf/sphRefinement.py:136-190) on the device-resident state: the fluid
 * particles mask (caller order, n bytes) selects each become 2^dim daughters, the first in place
 * and the rest appended in the caller's order.  *split returns how many split. */
int sph_split(SphSystem *sys, const uint8_t *mask, double reference_density, double length_ratio, int64_t *split);

/* mergeParticles (src/pysurf/sphRefinement.py:219-311; WcsphSolver.merge, src/pysurf/sphSolver.py:2046-2092)
 * on the device-resident state: the split fluid particles mask (caller order, n bytes) selects merge,
 * 2^dim of one level into one particle of the level above (cubes one coarser particle across,
 * two passes, the 2^dim nearest each cube's centre); the merged particle takes its group's first
 * place, and fluid from the end fills the places the others leave among the boundary's.  *groups
 * and *removed_energy (the members' kinetic energy about their centres of mass) come back, and
 * source, when not NULL, takes the caller index before the merge of each particle after (the new
 * count of entries, sph_count).  Refused with particle shifting on.  When too few fluid particles follow
 * the boundary in caller order to fill the places a merge leaves among it, the call fails
 * (SPH_ERR_CUDA, as the reference raises) and the state is as it was. */
int sph_merge(SphSystem *sys, const uint8_t *mask, double reference_density, double reference_mass,
              double length_ratio, int64_t *groups, double *removed_energy, int64_t *source);

/* Crest-zone refinement on the device: every fluid particle of mass at least min_mass (one not yet
 * split) whose column -- columns `width` across from (x0, y0), nx by ny of them (ny 1 in 2D) --
 * has its highest fluid particle above `threshold` (the surface's height), splits as sph_split
 * splits it; *split gets how many did.  The zone of BreakingWave3D._refineCrest
 * (src/pysurf/BreakingWave3D.py:530-576) read as the columns where the surface stands high. */
int sph_split_crest_zone(SphSystem *sys, double x0, double y0, double width, int64_t nx, int64_t ny,
                         double threshold, double min_mass, double reference_density, double length_ratio,
                         int64_t *split);

/* ---- The breaking tracker's reads of the fluid (2D) -----------------------------------------
 *
 * The reference's BreakingTracker (src/pysurf/waveBreaking.py:709-906) reads the fluid's pulled
 * positions every 0.01 sqrt(d / g) of simulated time (src/pysurf/BreakingWave.py:885-912).  These
 * replace that pull with the three small things an update needs, computed on the device with the
 * reference's float64 arithmetic term by term, so they equal the host's reads of pulled positions.
 *
 * sph_surface_tops: tops[c] = the largest height of a fluid particle in column
 *   floor((x - x0) / width) = c, c < count; -inf for an empty column (freeSurfaceProfile,
 *   src/pysurf/waveBreaking.py:129-162, before its half-column offset).
 * sph_face_cells: marks (bands rows of columns bytes) = 1 where a fluid particle with
 *   low_x <= x < high_x and z > low_z marks the cell (band0 + db, column0 + dc), db, dc in {0, 1},
 *   column0 = floor((x - half - start) / spacing), band0 = floor((z - half - base) / spacing)
 *   (frontFaceLean's occupancy, src/pysurf/waveBreaking.py:559-634).
 * sph_bed_sheet: the x of every fluid particle less than wet_height above the bed profile
 *   (bed_x, bed_z; numpy.interp between its vertices), in no set order, into xs (capacity
 *   entries; *count gets how many there are) (waterlineX, src/pysurf/waveBreaking.py:636-656). */
int sph_surface_tops(SphSystem *sys, double x0, double width, int64_t count, double *tops);
int sph_face_cells(SphSystem *sys, double low_x, double high_x, double low_z, double half, double start,
                   double base, double spacing, int64_t columns, int64_t bands, uint8_t *marks);
int sph_bed_sheet(SphSystem *sys, const double *bed_x, const double *bed_z, int64_t bed_count, double wet_height,
                  double *xs, int64_t capacity, int64_t *count);
/* The same three reads in 3D over one section of the tank (BreakingWave3D._readSections,
 * src/pysurf/BreakingWave3D.py:461-480): the fluid whose y lies within half_width of y
 * (|y_p - y| < half_width, the reference's section mask), read in its (x, z) plane, z the
 * vertical; the arguments otherwise as above.  SPH_ERR_UNSUPPORTED in 2D, as the reads above are
 * in 3D. */
int sph_section_tops(SphSystem *sys, double y, double half_width, double x0, double width, int64_t count, double *tops);
int sph_section_face_cells(SphSystem *sys, double y, double half_width, double low_x, double high_x, double low_z,
                           double half, double start, double base, double spacing, int64_t columns, int64_t bands,
                           uint8_t *marks);
int sph_section_bed_sheet(SphSystem *sys, double y, double half_width, const double *bed_x, const double *bed_z,
                          int64_t bed_count, double wet_height, double *xs, int64_t capacity, int64_t *count);

/* The same loop in three calls, for callers that overlap their own work with the steps:
 * sph_begin_steps sets the clock and the limits on the device; sph_enqueue_steps queues `count`
 * steps on the handle's stream and returns at once (steps past the limits do nothing);
 * sph_finish_steps waits and reads the clock back. */
int sph_begin_steps(SphSystem *sys, double time, int64_t step, double last_dt, double until_time, int64_t max_step,
                    double shortest_length, double cfl, double max_time_step, int64_t filter_interval);
int sph_enqueue_steps(SphSystem *sys, int64_t count);
int sph_finish_steps(SphSystem *sys, double *time, int64_t *step, double *last_dt);

/* Timing of the last sph_advance call (milliseconds, device events), and of each stage of the
 * last step that ran (cells, filter, wall, gradients, momentum, kick, continuity: *count of them,
 * named by sph_stage_name), and the kernels one step launches. */
int sph_last_advance_ms(const SphSystem *sys, double *ms);
int sph_stage_times(SphSystem *sys, double *ms, int64_t capacity, int64_t *count);
const char *sph_stage_name(int64_t stage);
int sph_step_launches(SphSystem *sys, int64_t *kernels);

/* ---- For callers that cannot allocate device memory ----------------------------------------
 *
 * No counterpart in the reference.  Callers whose device memory is all owned by their own pool
 * allocator, or whose loop must not enter the CUDA allocator while it runs, cannot let the library
 * cudaMalloc.  This entry point allocates nothing: its inputs and output are the caller's device
 * arrays, and its scratch is a fixed 64 KiB + 256 B file-scope device array that every GPU loading
 * the library holds until exit.  It is the momentum sweep's closing reduction on its own: the
 * largest fluid speed (float64) and acceleration (float32 length), and the time step from them
 * (cflTimeStep, src/pysurf/sphSolver.py:1410-1424), written to out[0..2] on the device.
 * velocities and accelerations are (n, dim) float64, is_fluid n bytes; stream a cudaStream_t or
 * NULL.  It returns once the work is queued.  At most 16,777,216 particles: more is refused with
 * SPH_ERR_INVALID before any launch.  The first call on a device looks the scratch's address up
 * with that device current; make it before any stream capture begins.  Calls share the scratch:
 * calls that overlap on the GPU race and must not be made. */
int sph_fluid_maxima_noalloc(const double *velocities, const double *accelerations, const uint8_t *is_fluid,
                             int64_t n, int dimensions, double smoothing_length, double sound_speed, double cfl,
                             double max_time_step, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PYSURF_B200_H */
