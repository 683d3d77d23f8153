/*
 * softbox_b200.h — C ABI of the B200 rigid-rod mechanics library (libsoftbox_b200.so).
 *
 * Drop-in boundary: each entry point below replaces the body of one public static
 * method of the reference's System classes (package softbox/, notaboxllc/SoftBox). The
 * Java side keeps its signatures and its planar SoA store layouts
 * ([x0..xN-1 | y0..yN-1 | z0..zN-1], FilamentStore.java:10-22) and calls these
 * functions through the Foreign Function & Memory API (a MethodHandle downcall per entry
 * point, with MemorySegment addresses for the device pointers). Conventions:
 *   - every array argument is a DEVICE pointer owned by the caller (the store);
 *     entry points allocate nothing except where a comment says "scratch";
 *   - an argument `n`, `cap`, ... carries the length the Java code reads with
 *     getSize() (divided by 3 for planar vectors);
 *   - small parameter arrays (params, counts, kinParams, ...) are device arrays with
 *     the reference's documented slot layout, exactly like the TornadoVM buffers;
 *   - every call is asynchronous on the context's stream; results are ordered by
 *     that stream; errors are returned as sbx_status and described by
 *     sbx_ctx_last_error(). No C++ exception crosses this boundary.
 *   - a context is not thread-safe; use one per host thread.
 */
#ifndef SOFTBOX_B200_H
#define SOFTBOX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef int32_t sbx_status;
#define SBX_OK          0
#define SBX_EINVAL     -1   /* bad argument / size */
#define SBX_ECUDA      -2   /* CUDA runtime error */
#define SBX_EOVERFLOW  -3   /* a capacity (MAX_CAND, contents) was exceeded; counts continue past it */
#define SBX_ETIMEOUT   -4   /* a bounded device wait gave up */
#define SBX_ENOMEM     -5
#define SBX_ENONFINITE -6   /* a supplied-noise / state array holds NaN or Inf */
#define SBX_ESTATE     -7   /* call out of order (e.g. plan not built) */

/* reference constants (SpatialGrid.java:46-48, CrossBridgeSystem.java:36, ...) */
#define SBX_MAX_CAND        256
#define SBX_GRID_SCAN_CHUNK 512
#define SBX_XB_STRIDE        13
#define SBX_XL_STRIDE        12
#define SBX_MINI_STRIDE       6
#define SBX_STRAIN_WIN       10
#define SBX_TORQUE_WIN        5
#define SBX_FORCEDOT_WIN     10

typedef struct sbx_ctx sbx_ctx;

/* ---------------------------------------------------------------- context / memory */
/* Creates a context on `device`. `stream` is a cudaStream_t to run on, or NULL to
 * create a private blocking stream (ordered against the legacy default stream, and
 * capturable into CUDA graphs, which the legacy stream is not). */
sbx_status sbx_ctx_create(int device, void* stream, sbx_ctx** out);
sbx_status sbx_ctx_destroy(sbx_ctx* ctx);
const char* sbx_ctx_last_error(sbx_ctx* ctx);
sbx_status sbx_ctx_set_stream(sbx_ctx* ctx, void* stream);
void* sbx_ctx_stream(sbx_ctx* ctx);
/* Waits for the context's stream (and its copy stream, if it has one). Also reports (SBX_EINVAL, then cleared) an input that a
 * kernel since the last sync found outside its documented range and skipped: a CSR key at
 * or past its row count (sbx_csr_build*, sbx_grid_build); and (SBX_ETIMEOUT, then cleared) a
 * staged reach walk whose bulk copies did not complete in time. */
sbx_status sbx_ctx_sync(sbx_ctx* ctx);
/* number of kernels this context has launched (for launch accounting) */
int64_t sbx_ctx_launch_count(sbx_ctx* ctx);
/* bytes of device scratch the context holds (grows on demand, never shrinks; -1 for NULL) */
int64_t sbx_ctx_scratch_bytes(sbx_ctx* ctx);
/* 1 in the index-checking debug build (libsoftbox_b200_check.so, compiled with -DSBX_CHECK),
 * 0 in the normal build. */
int32_t sbx_check_build(void);
/* Index checks of the debug build: the number of data-dependent indices the kernels found
 * outside the array they index (and skipped) since the last reset, the first one's site
 * (1 chain neighbour, 2 bound segment, 3 link end, 4 CSR list entry, 5 grid cell, 6 motor
 * slot, 7 reach-walk entry, 8 CSR position; 0 when none) and its value; reset != 0 clears
 * them. Synchronous (reads device counters). The normal build reports zeros. */
sbx_status sbx_check_report(int64_t* count, int32_t* site, int64_t* index, int32_t reset);

/* DataTransferMode analogues: FIRST_EXECUTION / EVERY_EXECUTION uploads and
 * UNDER_DEMAND pulls are plain async copies on the context stream. */
sbx_status sbx_malloc(sbx_ctx* ctx, size_t bytes, void** dptr);
sbx_status sbx_free(sbx_ctx* ctx, void* dptr);
sbx_status sbx_upload(sbx_ctx* ctx, void* dst_dev, const void* src_host, size_t bytes);
sbx_status sbx_download(sbx_ctx* ctx, void* dst_host, const void* src_dev, size_t bytes);
/* The same copy without the wait: the bytes are on the host once the stream has passed it
 * (sbx_ctx_sync, or a marker recorded after it and waited for). */
sbx_status sbx_download_async(sbx_ctx* ctx, void* dst_host, const void* src_dev, size_t bytes);
/* Stream markers (slots 0..7): sbx_ctx_mark records the current end of the context's stream
 * in a slot; sbx_ctx_wait_mark waits until the stream has passed it and reports the kernels'
 * range errors like sbx_ctx_sync. A host can so keep the next step queued while it reads
 * the previous step's results. */
sbx_status sbx_ctx_mark(sbx_ctx* ctx, int32_t slot);
sbx_status sbx_ctx_wait_mark(sbx_ctx* ctx, int32_t slot);
/* A result copy off the context's stream: sbx_download_async_side queues the copy on the
 * context's copy stream (created on first use), after everything queued on its stream so
 * far, and returns; the stream moves on at once, so the copy overlaps the next uploads.
 * sbx_ctx_mark_side records the copy stream's current end in a marker slot (wait for it on
 * the host with sbx_ctx_wait_mark); sbx_ctx_stream_wait_mark makes work queued later on the
 * context's stream start after a marker, e.g. a step that overwrites the copied array.
 * sbx_ctx_mark_side before any side copy: SBX_EINVAL; so is a wait on an unrecorded slot. */
sbx_status sbx_download_async_side(sbx_ctx* ctx, void* dst_host, const void* src_dev, size_t bytes);
sbx_status sbx_ctx_mark_side(sbx_ctx* ctx, int32_t slot);
sbx_status sbx_ctx_stream_wait_mark(sbx_ctx* ctx, int32_t slot);
sbx_status sbx_memset(sbx_ctx* ctx, void* dst_dev, int value, size_t bytes);

/* ---------------------------------------------------------------- drag (host-init systems, run on device)
 * DragTensorSystem.run(FilamentStore) (DragTensorSystem.java:71-97); `aeta` is the
 * viscosity in Pa*s (the reference reads Constants.aeta = 0.1). */
sbx_status sbx_drag_run_filament(sbx_ctx* ctx, int32_t n, const int32_t* monomerCount,
                                 const int32_t* end1NbrSlot, const int32_t* end2NbrSlot, double aeta,
                                 float* segLength, float* bTransGam, float* bRotGam,
                                 float* bTransDiff, float* bRotDiff);
/* DragTensorSystem.run(MotorStore) (DragTensorSystem.java:105-122) */
sbx_status sbx_drag_run_motor(sbx_ctx* ctx, int32_t nMotors, double aeta, float* segLength,
                              float* bTransGam, float* bRotGam, float* bTransDiff, float* bRotDiff);
/* MiniFilamentStore.initBackboneDrag (MiniFilamentStore.java:121-134); backbone length is a parameter */
sbx_status sbx_drag_run_backbone(sbx_ctx* ctx, int32_t nBb, double bbLenUm, double aeta, float* segLength,
                                 float* bTransGam, float* bRotGam, float* bTransDiff, float* bRotDiff,
                                 float* bbInvDragY);

/* ---------------------------------------------------------------- Brownian forcing
 * BrownianForceSystem.brownianForce (BrownianForceSystem.java:44-106): Wang-hash keyed
 * (slot, counts[1]=step, counts[2]=seed), three Box-Muller pairs. params[1]=sqrt(2kT/dt). */
sbx_status sbx_brownian_force(sbx_ctx* ctx, int32_t n, float* randForce, float* randTorque,
                              const float* bTransGam, const float* bRotGam, const float* brownTransScale,
                              const float* brownRotScale, const float* params, const int32_t* counts);
/* Same amplitude law with Philox4x32-10 keyed (seed64, step, slot). */
sbx_status sbx_brownian_force_philox(sbx_ctx* ctx, int32_t n, float* randForce, float* randTorque,
                                     const float* bTransGam, const float* bRotGam,
                                     const float* brownTransScale, const float* brownRotScale,
                                     const float* params, const int32_t* counts, uint64_t seed);
/* Supplied-noise mode: noise is planar [6][n] (gfx|gfy|gfz|gtx|gty|gtz) standard normals.
 * Returns SBX_ENONFINITE (and writes nothing) if any entry is NaN/Inf. */
sbx_status sbx_brownian_force_supplied(sbx_ctx* ctx, int32_t n, float* randForce, float* randTorque,
                                       const float* bTransGam, const float* bRotGam,
                                       const float* brownTransScale, const float* brownRotScale,
                                       const float* params, const float* noise);

/* ChainBendingForceSystem.zeroAccumulators (ChainBendingForceSystem.java:38-45) */
sbx_status sbx_zero_accumulators(sbx_ctx* ctx, int32_t n, float* forceSum, float* torqueSum);

/* ---------------------------------------------------------------- integration
 * RigidRodLangevinIntegrationSystem.integrate (RigidRodLangevinIntegrationSystem.java:33-112).
 * coord64 may be NULL; when given, centres accumulate in FP64 and coord receives the
 * rounded projection (the per-step increment is the reference's FP32 dt*v). */
sbx_status sbx_integrate(sbx_ctx* ctx, int32_t n, float* coord, double* coord64, float* uVec, float* yVec,
                         const float* forceSum, const float* torqueSum, const float* randForce,
                         const float* randTorque, const float* bTransGam, const float* bRotGam,
                         const float* params);
/* DerivedGeometrySystem.derive (DerivedGeometrySystem.java:27-73) */
sbx_status sbx_derive(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec, float* yVec,
                      float* zVec, float* end1, float* end2, const float* segLength);
/* ContainmentSystem.confine (ContainmentSystem.java:58-126); boxParams[0..6] */
sbx_status sbx_confine(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                       const float* segLength, const float* bTransGam, float* forceSum, float* torqueSum,
                       const float* boxParams, const int32_t* counts);
/* MechanicsFusion.forceBuild / integDerive / integDeriveConfined (MechanicsFusion.java:52-338) */
sbx_status sbx_fusion_force_build(sbx_ctx* ctx, int32_t n, float* forceSum, float* torqueSum,
                                  float* randForce, float* randTorque, const float* bTransGam,
                                  const float* bRotGam, const float* brownTransScale,
                                  const float* brownRotScale, const float* params, const int32_t* counts);
sbx_status sbx_fusion_integ_derive(sbx_ctx* ctx, int32_t n, float* coord, double* coord64, float* uVec,
                                   float* yVec, float* zVec, const float* segLength, float* end1, float* end2,
                                   const float* forceSum, const float* torqueSum, const float* randForce,
                                   const float* randTorque, const float* bTransGam, const float* bRotGam,
                                   const float* params);
sbx_status sbx_fusion_integ_derive_confined(sbx_ctx* ctx, int32_t n, float* coord, double* coord64,
                                            float* uVec, float* yVec, float* zVec, const float* segLength,
                                            float* end1, float* end2, float* forceSum, float* torqueSum,
                                            const float* randForce, const float* randTorque,
                                            const float* bTransGam, const float* bRotGam,
                                            const float* boxParams, const int32_t* counts);

/* ---------------------------------------------------------------- chain
 * ChainBendingForceSystem.chainForces (ChainBendingForceSystem.java:105-331) */
sbx_status sbx_chain_forces(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                            const float* segLength, const int32_t* end2NbrSlot, const int32_t* end2NbrSide,
                            const int32_t* end1NbrSlot, const int32_t* end1NbrSide, const float* bTransGam,
                            const float* bRotGam, float* forceSum, float* torqueSum, const float* chainParams);
/* chainForces followed, in the same pass, by the filament-side gathers of the step in the
 * reference's order: CrosslinkerSystem.segGatherA, segGatherB (CrosslinkerSystem.java:129-173)
 * and CrossBridgeSystem.segGather (CrossBridgeSystem.java:302-320), each reading the
 * row-ordered payload of sbx_csr_build_payload (xlinkData offsets 0 / 6 guarded by linkState;
 * bondData offset 6). The accumulators get the bits of sbx_chain_forces followed by the three
 * separate gathers. A null offsets pointer skips that gather. */
sbx_status sbx_fusion_chain_gathers(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                                    const float* segLength, const int32_t* end2NbrSlot,
                                    const int32_t* end2NbrSide, const int32_t* end1NbrSlot,
                                    const int32_t* end1NbrSide, const float* bTransGam, const float* bRotGam,
                                    float* forceSum, float* torqueSum, const float* chainParams,
                                    const int32_t* segOffsetsA, const float* rowPayloadA,
                                    const int32_t* segOffsetsB, const float* rowPayloadB,
                                    const int32_t* segMotorOffsets, const float* rowPayloadM);

/* ---------------------------------------------------------------- body view publishing
 * FilamentStore.publishToBodyView (FilamentStore.java:275-328); filState may be NULL (8-arg form) */
sbx_status sbx_filament_publish(sbx_ctx* ctx, int32_t n, const float* coord, const float* segLength,
                                int32_t cap, float* center, float* boundingRadius, int32_t* ownerStore,
                                int32_t* ownerSlot, const float* viewParams, const int32_t* filState);
/* MotorStore.publishHeadFromBody (MotorStore.java:300-314) */
sbx_status sbx_motor_publish_head(sbx_ctx* ctx, int32_t nMotors, const float* bodyCoord,
                                  const float* bodyUVec, const float* bodySegLength, float* head,
                                  float* uVec, float* rodUVec);
/* MotorStore.publishToBodyView (MotorStore.java:326-347); publishParams[0] = base slot */
sbx_status sbx_motor_publish(sbx_ctx* ctx, int32_t nMotors, const float* head, const float* reach,
                             int32_t cap, float* center, float* boundingRadius, int32_t* ownerStore,
                             int32_t* ownerSlot, const int32_t* publishParams);

/* ---------------------------------------------------------------- spatial grid
 * SpatialGrid.bodyCell (SpatialGrid.java:51-75); counts[1] = S */
sbx_status sbx_grid_body_cell(sbx_ctx* ctx, int32_t cap, const float* center, const float* gridParams,
                              const int32_t* gridDims, const int32_t* counts, int32_t* bodyCell);
/* The counting sort that replaces gridZero+gridHistogram+gridScanLocal/Chunks/Add+gridScatter
 * (SpatialGrid.java:78-182) and the chunked gridChunk* variant (SpatialGrid.java:237-331):
 * atomic cell histogram, block scan over GRID_SCAN_CHUNK tiles (chunkSum holds the tile
 * sums, as in the reference), scatter, then an in-cell ascending sort so that the
 * within-cell order is body-index order. Outputs equal the serial reference bit for bit:
 * gridCellOffsets[0..totalCells] (terminator clamped to contentsCap), gridCellContents,
 * cellCount (= per-cell counts, as the serial gridScatter leaves it), chunkSum.
 * `cap` is the length of bodyCell; contentsCap < cap is rejected (the reference sizes
 * gridCellContents = cap). Uses context scratch (cap ints) for the unordered scatter. */
sbx_status sbx_grid_build(sbx_ctx* ctx, int32_t cap, const int32_t* bodyCell, const int32_t* counts,
                          int32_t totalCells, int32_t* cellCount, int32_t* chunkSum,
                          int32_t* gridCellOffsets, int32_t* gridCellContents, int32_t contentsCap);
/* SpatialGrid.broadPhase (SpatialGrid.java:340-406); candPartner is cap*SBX_MAX_CAND */
sbx_status sbx_grid_broad_phase(sbx_ctx* ctx, int32_t cap, const float* center, const float* boundingRadius,
                                const int32_t* bodyCell, const int32_t* gridCellOffsets,
                                const int32_t* gridCellContents, const int32_t* gridDims,
                                const float* gridParams, const int32_t* counts, int32_t* candPartner,
                                int32_t* candCount);
/* SpatialGrid.bruteForce (SpatialGrid.java:413-445) */
sbx_status sbx_grid_brute_force(sbx_ctx* ctx, int32_t cap, const float* center, const float* boundingRadius,
                                const float* gridParams, const int32_t* counts, int32_t* brutePartner,
                                int32_t* bruteCount);

/* ---------------------------------------------------------------- binding / unbinding
 * BindingDetectionSystem.gridReachable (BindingDetectionSystem.java:143-228); nM = counts[0] */
sbx_status sbx_binding_grid_reachable(sbx_ctx* ctx, const float* head, const float* uVec, const float* rodUVec,
                                      int32_t nSeg, const float* segEnd1, const float* segEnd2,
                                      const float* gridParams, const int32_t* gridDims,
                                      const int32_t* gridCellOffsets, const int32_t* gridCellContents,
                                      const int32_t* ownerStore, const int32_t* ownerSlot,
                                      int32_t* motorReachSeg, int32_t* motorReachCount,
                                      const float* kinParams, int32_t nM);
/* gridReachable over cell-ordered segment endpoints: sbx_grid_cell_endpoints writes, for every
 * grid entry idx < gridCellOffsets[totalCells], cellEnd1[4 idx..] = (end1 xyz, slot as int
 * bits; -1 for a non-filament entry) and cellEnd2[4 idx..] = (end2 xyz, 0) (cap float4 each,
 * 16-byte aligned); sbx_fusion_grid_reachable then walks them with the reach lists and
 * counts of sbx_binding_grid_reachable. */
sbx_status sbx_grid_cell_endpoints(sbx_ctx* ctx, int32_t cap, int32_t totalCells,
                                   const int32_t* gridCellOffsets, const int32_t* gridCellContents,
                                   const int32_t* ownerStore, const int32_t* ownerSlot, int32_t nSeg,
                                   const float* segEnd1, const float* segEnd2, float* cellEnd1, float* cellEnd2);
sbx_status sbx_fusion_grid_reachable(sbx_ctx* ctx, const float* head, const float* uVec, const float* rodUVec,
                                     const float* gridParams, const int32_t* gridDims,
                                     const int32_t* gridCellOffsets, const float* cellEnd1,
                                     const float* cellEnd2, int32_t* motorReachSeg, int32_t* motorReachCount,
                                     const float* kinParams, int32_t nM);
/* The same walk (same reach lists and counts) with each tile of 64 x-cells of one y-row,
 * every z, handled by one block that stages the tile's neighbourhood in shared memory: the
 * cell offsets of the 3*nZ rows around it and their cell-ordered endpoint pairs (bulk copies);
 * the heads binned in the tile then walk shared memory. Takes the grid dimensions on the
 * host, the grid contents and owners (to find the tile's heads), bodyCell, cap and
 * publishParams (heads in no cell take the plain walk). nZ > 16 falls back to
 * sbx_fusion_grid_reachable. A bulk-copy wait past one second is reported as SBX_ETIMEOUT by
 * the next sbx_ctx_sync (the tile's heads then take the plain walk). */
sbx_status sbx_fusion_grid_reachable_staged(sbx_ctx* ctx, const float* head, const float* uVec,
                                            const float* rodUVec, const float* gridParams,
                                            const int32_t* gridDims, int32_t nX, int32_t nY, int32_t nZ,
                                            const int32_t* gridCellOffsets, const int32_t* gridCellContents,
                                            const int32_t* ownerStore, const int32_t* ownerSlot,
                                            const int32_t* bodyCell, int32_t cap, const int32_t* publishParams,
                                            const float* cellEnd1, const float* cellEnd2, int32_t* motorReachSeg,
                                            int32_t* motorReachCount, const float* kinParams, int32_t nM);
/* BindingDetectionSystem.bruteReachable (BindingDetectionSystem.java:260-283) */
sbx_status sbx_binding_brute_reachable(sbx_ctx* ctx, const float* head, const float* uVec,
                                       const float* rodUVec, int32_t nSeg, const float* segEnd1,
                                       const float* segEnd2, int32_t* reachSeg, int32_t* reachCount,
                                       const float* kinParams, int32_t nM);
/* BindingDetectionSystem.bindNearest (BindingDetectionSystem.java:356-389) */
sbx_status sbx_binding_bind_nearest(sbx_ctx* ctx, const float* head, const float* uVec, const float* rodUVec,
                                    int32_t nSeg, const float* segEnd1, const float* segEnd2,
                                    const int32_t* motorCandSeg, const int32_t* motorCandCount,
                                    int32_t* boundSeg, float* bindArc, const float* kinParams, int32_t nM);
/* NucleotideCycleSystem.catchSlipRelease (NucleotideCycleSystem.java:77-134) */
sbx_status sbx_nucleotide_release(sbx_ctx* ctx, int32_t nM, int32_t* boundSeg, const float* forceDotFil,
                                  const float* forceMag, int32_t* cooldown, int32_t* stats,
                                  int32_t* capStats, const float* kinParams, const int32_t* counts);
/* NucleotideCycleSystem.cycle (NucleotideCycleSystem.java:33-69) */
sbx_status sbx_nucleotide_cycle(sbx_ctx* ctx, int32_t nM, int32_t* nucleotideState, const int32_t* boundSeg,
                                const float* forceDotHist, const float* nucParams, const int32_t* counts);

/* ---------------------------------------------------------------- cross-bridge
 * CrossBridgeSystem.bondForces / applyHeadForce / registerForceDot (CrossBridgeSystem.java:58-187) */
sbx_status sbx_xbridge_bond_forces(sbx_ctx* ctx, int32_t nB, const float* motorCoord, const float* motorUVec,
                                   const float* motorYVec, const float* motorBRotGam, int32_t nSeg,
                                   const float* filCoord, const float* filUVec, const float* filYVec,
                                   const float* filBRotGam, const float* filSegLength, const int32_t* boundSeg,
                                   const float* bindArc, const int32_t* nucleotideState, float* bondData,
                                   const float* xbParams);
sbx_status sbx_xbridge_apply_head_force(sbx_ctx* ctx, int32_t nB, const float* bondData,
                                        float* bodyForceSum, float* bodyTorqueSum);
sbx_status sbx_xbridge_register_force_dot(sbx_ctx* ctx, int32_t nM, const float* bondData,
                                          const int32_t* boundSeg, float* forceDotFil, float* forceMag,
                                          float* forceDotHist, int32_t* forceDotPlace);
/* The CSR-inverse that replaces csrHistogram/csrScan/csrScatter and csrChunk*
 * (CrossBridgeSystem.java:190-298): rows = key values, items in ascending index per row.
 * Outputs equal the serial reference: rowOffsets[0..nRows], rowList, rowCount (= row
 * lengths, as the serial csrScatter leaves it). Uses context scratch for the scan.
 * Keys: -1 (or any negative value) = unbound item, skipped as in the reference; 0..nRows-1
 * = its row. A key >= nRows (where the reference's Java would throw) is skipped too and
 * reported by the next sbx_ctx_sync as SBX_EINVAL; the outputs then hold the valid items. */
sbx_status sbx_csr_build(sbx_ctx* ctx, const int32_t* keys, int32_t nItems, int32_t nRows,
                         int32_t* rowCount, int32_t* rowOffsets, int32_t* rowList);
/* No counterpart in the reference. Same outputs as sbx_csr_build, but it allocates no
 * device memory: its scratch is a fixed array inside the library (about 4 MB per device),
 * for callers that cannot let a call allocate or synchronise (a host that owns the device
 * heap under a fixed budget, a step sequence that must not stall). Inputs above
 * SBX_CSR_NOALLOC_MAX_ITEMS items or SBX_CSR_NOALLOC_MAX_ROWS rows return SBX_EINVAL.
 * Nothing needs to start at zero. The scratch is shared by every context on a device:
 * calls that overlap in time on one device (different streams) race; calls on one stream
 * are safe. The first call on each device sets the scratch up; make it before any stream
 * capture begins. Keys as for sbx_csr_build. */
#define SBX_CSR_NOALLOC_MAX_ITEMS (1 << 20)
#define SBX_CSR_NOALLOC_MAX_ROWS (1 << 22)
sbx_status sbx_csr_build_noalloc(sbx_ctx* ctx, const int32_t* keys, int32_t nItems, int32_t nRows,
                                 int32_t* rowCount, int32_t* rowOffsets, int32_t* rowList);
/* sbx_csr_build that also copies each item's 6-float payload (payload[item * payloadStride +
 * payloadOffset + 0..5]; zeros where guard != NULL and guard[item] < 0) into rowPayload in
 * list order: row r's items are rowPayload[6 k .. 6 k + 5] for k in [rowOffsets[r],
 * rowOffsets[r+1]). rowPayload: 6 * nItems floats, 8-byte aligned. */
sbx_status sbx_csr_build_payload(sbx_ctx* ctx, const int32_t* keys, int32_t nItems, int32_t nRows,
                                 int32_t* rowCount, int32_t* rowOffsets, int32_t* rowList,
                                 const float* payload, int32_t payloadStride, int32_t payloadOffset,
                                 const int32_t* guard, float* rowPayload);
/* CrossBridgeSystem.segGather (CrossBridgeSystem.java:302-320) */
sbx_status sbx_xbridge_seg_gather(sbx_ctx* ctx, int32_t nSeg, const int32_t* segMotorOffsets,
                                  const int32_t* segMotorMyo, const float* bondData, float* filForceSum,
                                  float* filTorqueSum);
/* CrossBridgeSystem.bruteGather (CrossBridgeSystem.java:323-337) */
sbx_status sbx_xbridge_brute_gather(sbx_ctx* ctx, int32_t nSeg, int32_t nM, const int32_t* boundSeg,
                                    const float* bondData, float* bForceSum, float* bTorqueSum);

/* ---------------------------------------------------------------- crosslinkers
 * CrosslinkerSystem.linkForces / segGatherA / segGatherB / bruteGather / unbind /
 * countActiveLinks / linkTorsion (CrosslinkerSystem.java:51-281, 694-808) */
sbx_status sbx_xlink_count_active(sbx_ctx* ctx, int32_t nLinks, const int32_t* linkState,
                                  const int32_t* linkFilA, const int32_t* linkFilB, int32_t nSeg,
                                  int32_t* activeLinkCount);
sbx_status sbx_xlink_forces(sbx_ctx* ctx, int32_t nSeg, const float* filCoord, const float* filUVec,
                            const float* filEnd1, const float* filBTransGam, int32_t nLinks,
                            const int32_t* linkFilA, const int32_t* linkFilB, const float* loc1,
                            const float* loc2, const int32_t* filLinkCt, float* xlinkData,
                            const float* xlParams);
sbx_status sbx_xlink_torsion(sbx_ctx* ctx, int32_t nSeg, const float* filUVec, int32_t nLinks,
                             const int32_t* linkFilA, const int32_t* linkFilB, const int32_t* linkState,
                             const int32_t* linkOrientSame, float* torqueMagHist, int32_t* torqueMagPlace,
                             float* xlinkData, const float* torsionParams);
/* side = 0 gathers the A-side payload [0..5], side = 1 the B-side payload [6..11] */
sbx_status sbx_xlink_seg_gather(sbx_ctx* ctx, int32_t side, int32_t nSeg, const int32_t* segOffsets,
                                const int32_t* segLinkIdx, const float* xlinkData, const int32_t* linkState,
                                float* filForceSum, float* filTorqueSum);
sbx_status sbx_xlink_brute_gather(sbx_ctx* ctx, int32_t nSeg, int32_t nLinks, const int32_t* linkFilA,
                                  const int32_t* linkFilB, const float* xlinkData, const int32_t* linkState,
                                  float* bForceSum, float* bTorqueSum);
sbx_status sbx_xlink_unbind(sbx_ctx* ctx, int32_t nSeg, const float* filUVec, const float* filEnd1,
                            int32_t nLinks, const int32_t* linkFilA, const int32_t* linkFilB,
                            const float* loc1, const float* loc2, int32_t* linkState, float* strainHist,
                            int32_t* strainPlace, const float* offParams, const int32_t* counts);

/* ---------------------------------------------------------------- crosslinker formation + allocator
 * CrosslinkerSystem formation (CrosslinkerSystem.java:405-756) and the scan-rank free-list
 * allocator (:297-345). formParams: [0] maxXLinkBondAngle (rad) [1] crossLinkGrabDist^2
 * [2] minSepBetweenXLinks [3] maxXLinksOnSeg [4] P_form [5] loc jitter half-range
 * [6] crossLinkGrabDist; formCounts: [0] nCand (written) [1] step [2] seed [3] xLinkMode
 * (0 both, 1 parallel, -1 antiparallel) (CrosslinkerStore.java:108-112). The formation grid
 * (FormationGrid.java) is built with sbx_filament_publish + sbx_grid_body_cell + sbx_grid_build. */
/* filFilCandidates (:431-452): all cross-filament pairs i<j within the coarse capsule bound,
 * lexicographic, capped at reqCap, unused tail keyed -1. Uses context scratch. */
sbx_status sbx_xlink_fil_fil_candidates(sbx_ctx* ctx, int32_t nSeg, const float* coord, const float* segLength,
                                        const int32_t* filID, int32_t reqCap, int32_t* reqFilA, int32_t* reqFilB,
                                        const float* formParams, int32_t* formCounts);
/* gridFormCount (:474-516): per segment, partners j>i in its 27 formation-grid cells (<= 256) */
sbx_status sbx_xlink_grid_form_count(sbx_ctx* ctx, int32_t nSeg, const float* coord, const float* segLength,
                                     const int32_t* filID, const float* gridParams, const int32_t* gridDims,
                                     const int32_t* gridCellOffsets, const int32_t* gridCellContents,
                                     int32_t* candCountSeg, const float* formParams);
/* gridFormScan (:520-532): candBaseSeg = exclusive prefix (candBaseSeg[nSeg] = total),
 * formCounts[0] = min(total, reqCap), unused tail keyed -1. Uses context scratch. */
sbx_status sbx_xlink_grid_form_scan(sbx_ctx* ctx, int32_t nSeg, const int32_t* candCountSeg, int32_t* candBaseSeg,
                                    int32_t reqCap, int32_t* reqFilA, int32_t* reqFilB, int32_t* formCounts);
/* gridFormEmit (:538-595): partners ascending into each segment's region (== filFilCandidates) */
sbx_status sbx_xlink_grid_form_emit(sbx_ctx* ctx, int32_t nSeg, const float* coord, const float* segLength,
                                    const int32_t* filID, const float* gridParams, const int32_t* gridDims,
                                    const int32_t* gridCellOffsets, const int32_t* gridCellContents,
                                    const int32_t* candBaseSeg, const int32_t* candCountSeg, int32_t reqCap,
                                    int32_t* reqFilA, int32_t* reqFilB, const float* formParams);
/* formGates (:600-665): alignment, closest approach, loc + jitter, P_form -> gatePass, reqLoc1/2, reqOrient */
sbx_status sbx_xlink_form_gates(sbx_ctx* ctx, int32_t nSeg, const float* filUVec, const float* filEnd1,
                                const float* filEnd2, const float* filSegLength, int32_t reqCap,
                                const int32_t* reqFilA, const int32_t* reqFilB, float* reqLoc1, float* reqLoc2,
                                int32_t* reqOrient, int32_t* gatePass, const float* formParams,
                                const int32_t* formCounts);
/* formAdmitReduce (:670-682): per segment, the minimum gate-passing candidate index (sentinel reqCap) */
sbx_status sbx_xlink_form_admit_reduce(sbx_ctx* ctx, int32_t reqCap, const int32_t* reqFilA, const int32_t* reqFilB,
                                       const int32_t* gatePass, int32_t nSeg, int32_t* minCand);
/* formAdmit (:713-735): one new link per segment, saturation and spacing vs start-of-step links */
sbx_status sbx_xlink_form_admit(sbx_ctx* ctx, int32_t reqCap, const int32_t* reqFilA, const int32_t* reqFilB,
                                const float* reqLoc1, const float* reqLoc2, const int32_t* gatePass,
                                const int32_t* minCand, const int32_t* activeLinkCount, int32_t nLinks,
                                const int32_t* linkState, const int32_t* linkFilA, const int32_t* linkFilB,
                                const float* loc1, const float* loc2, int32_t* acceptFlag, const float* formParams);
/* freeFlags (:297-302): freeCount[s] = linkState[s] < 0 */
sbx_status sbx_xlink_free_flags(sbx_ctx* ctx, int32_t C, const int32_t* linkState, int32_t* freeCount);
/* CrossBridgeSystem.csrScan (CrossBridgeSystem.java:198-205): offsets = exclusive prefix of
 * counts, offsets[n] = total, counts reset to 0. Uses context scratch. */
sbx_status sbx_csr_scan(sbx_ctx* ctx, int32_t n, int32_t* counts, int32_t* offsets);
/* freeScatter (:306-314): freeList[freeOffsets[s]] = s for each FREE slot */
sbx_status sbx_xlink_free_scatter(sbx_ctx* ctx, int32_t C, const int32_t* linkState, const int32_t* freeOffsets,
                                  int32_t* freeList);
/* allocate (:322-341): accepted request r claims freeList[rankOffsets[r]] (below nFree) */
sbx_status sbx_xlink_allocate(sbx_ctx* ctx, int32_t K, const int32_t* reqFilA, const int32_t* reqFilB,
                              const float* reqLoc1, const float* reqLoc2, const int32_t* rankOffsets,
                              const int32_t* freeList, const int32_t* freeOffsets, int32_t C, int32_t* linkFilA,
                              int32_t* linkFilB, float* loc1, float* loc2, int32_t* linkState, float* strainHist,
                              int32_t* strainPlace);
/* placeOrient (:740-752): orientSame and a fresh torsion ring in each claimed slot */
sbx_status sbx_xlink_place_orient(sbx_ctx* ctx, int32_t K, const int32_t* reqOrient, const int32_t* rankOffsets,
                                  const int32_t* freeList, const int32_t* freeOffsets, int32_t C,
                                  int32_t* linkOrientSame, float* torqueMagHist, int32_t* torqueMagPlace);

/* ---------------------------------------------------------------- actin turnover
 * Planar filament slot arrays of capacity C (FilamentStore: coord/uVec/yVec [3*C], filState
 * FREE -1 / ACTIVE 0, end1/end2 neighbour slot and side). growCounts/depolyCounts carry
 * [1] step, [2] seed, [3] fires; severCounts/agingCounts carry [1] fires. Split and birth
 * requests use the crosslinker allocator's scan ranks: freeFlags/freeScatter on filState are
 * sbx_xlink_free_flags/_free_scatter (FilamentBirthSystem.java:41-58), ranks by sbx_csr_scan.
 * GrowthSystem.grow (GrowthSystem.java:73-104): barbed-tip growth, wang-hash salt "GROW";
 * growParams [P, halfmono, maxMon] */
sbx_status sbx_growth_grow(sbx_ctx* ctx, int32_t C, const int32_t* seedNode, int32_t* monomerCount, float* coord,
                           const float* uVec, int32_t* grewFlag, const float* growParams, const int32_t* growCounts);
/* GrowthSystem.markSplits (:106-136): split requests at splitThresh monomers, request index =
 * slot, request planar stride reqCap >= C; splitParams [halfmono, splitThresh, childMon] */
sbx_status sbx_growth_mark_splits(sbx_ctx* ctx, int32_t C, const int32_t* seedNode, const int32_t* monomerCount,
                                  const float* coord, const float* uVec, const float* yVec, int32_t* acceptFlag,
                                  float* reqCoord, float* reqUVec, float* reqYVec, int32_t reqCap,
                                  const float* splitParams, const int32_t* growCounts);
/* GrowthSystem.splitWire (:148-190): parent shrink and the 3-slot chain rewire per formed split */
sbx_status sbx_growth_split_wire(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                 const int32_t* freeList, const int32_t* freeOffsets, int32_t* monomerCount,
                                 float* coord, const float* uVec, int32_t* end1NbrSlot, int32_t* end1NbrSide,
                                 int32_t* end2NbrSlot, int32_t* end2NbrSide, int32_t* seedNode,
                                 const float* splitParams);
/* GrowthSystem.recomputeDrag (:199-228): segLength and slender-rod drag from monomerCount;
 * dragParams [halfmono, aeta, radius, kT, aPar, aOrth, aTurn, stdSeg, minMon] */
sbx_status sbx_growth_recompute_drag(sbx_ctx* ctx, int32_t C, const int32_t* monomerCount, float* segLength,
                                     const int32_t* end1NbrSlot, const int32_t* end2NbrSlot, float* bTransGam,
                                     float* bRotGam, float* bTransDiff, float* bRotDiff, const float* dragParams,
                                     const int32_t* growCounts);
/* DepolySystem.depoly (DepolySystem.java:70-101): pointed-tip loss at fixed rate, death below
 * the floor; depolyParams [P, halfmono, floor], salt "DEPO" */
sbx_status sbx_depoly(sbx_ctx* ctx, int32_t C, const int32_t* filState, int32_t* monomerCount, float* coord,
                      const float* uVec, const int32_t* end1NbrSlot, int32_t* returnedMon, int32_t* deathFlag,
                      const float* depolyParams, const int32_t* depolyCounts);
/* DepolySystem.depolyProxy (:115-145): rate = rateParams[0]*(1-fADP) + rateParams[1]*fADP */
sbx_status sbx_depoly_proxy(sbx_ctx* ctx, int32_t C, const int32_t* filState, int32_t* monomerCount, float* coord,
                            const float* uVec, const int32_t* end1NbrSlot, const float* nucFrac,
                            int32_t* returnedMon, int32_t* deathFlag, const float* depolyParams,
                            const float* depolyRateParams, const int32_t* depolyCounts);
/* DepolySystem.applyDeath (:158-188): free each dying slot and break its chain links */
sbx_status sbx_depoly_apply_death(sbx_ctx* ctx, int32_t C, int32_t* filState, int32_t* monomerCount,
                                  int32_t* seedNode, int32_t* end1NbrSlot, int32_t* end1NbrSide,
                                  int32_t* end2NbrSlot, int32_t* end2NbrSide, float* brownTransScale,
                                  float* brownRotScale, const int32_t* deathFlag);
/* SeveringSystem.cofilinAccumulate (SeveringSystem.java:37-49); cofilinParams [p_cof, ratio] */
sbx_status sbx_sever_cofilin_accumulate(sbx_ctx* ctx, int32_t C, const int32_t* filState, const float* nucFrac,
                                        float* cofFrac, const float* cofilinParams, const int32_t* severCounts);
/* SeveringSystem.cofilinDissolve (:58-74): death flags where cofFrac > ratio */
sbx_status sbx_sever_cofilin_dissolve(sbx_ctx* ctx, int32_t C, const int32_t* filState, const int32_t* monomerCount,
                                      const float* cofFrac, int32_t* severDeathFlag, int32_t* severReturnedMon,
                                      const float* cofilinParams, const int32_t* severCounts);
/* SeveringSystem.nucleateFreshCofilin (:88-98): cofFrac = 0 in each claimed slot */
sbx_status sbx_sever_nucleate_fresh_cofilin(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                            const int32_t* freeList, const int32_t* freeOffsets, float* cofFrac);
/* FilamentBirthSystem.allocate (FilamentBirthSystem.java:64-87): request pose into the claimed
 * slot, birthParams [brownTransScale, brownRotScale], state ACTIVE */
sbx_status sbx_birth_allocate(sbx_ctx* ctx, int32_t K, int32_t C, int32_t reqCap, const float* reqCoord,
                              const float* reqUVec, const float* reqYVec, const int32_t* rankOffsets,
                              const int32_t* freeList, const int32_t* freeOffsets, float* coord, float* uVec,
                              float* yVec, float* brownTransScale, float* brownRotScale, int32_t* filState,
                              const float* birthParams);
/* AgingSystem.age (AgingSystem.java:40-57): ATP -> ADP-Pi -> ADP; agingParams [pH, pD] */
sbx_status sbx_aging_age(sbx_ctx* ctx, int32_t C, const int32_t* filState, float* nucFrac,
                         const float* agingParams, const int32_t* agingCounts);
/* AgingSystem.growthAtp (:65-77): one fresh ATP monomer mixed into each grown tip */
sbx_status sbx_aging_growth_atp(sbx_ctx* ctx, int32_t C, const int32_t* grewFlag, const int32_t* monomerCount,
                                float* nucFrac);
/* AgingSystem.splitInheritNuc (:88-102): a split child takes its parent's fractions */
sbx_status sbx_aging_split_inherit_nuc(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                       const int32_t* freeList, const int32_t* freeOffsets, float* nucFrac);
/* AgingSystem.nucleateFreshAtp (:114-125): a newborn slot is all ATP */
sbx_status sbx_aging_nucleate_fresh_atp(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                        const int32_t* freeList, const int32_t* freeOffsets, float* nucFrac);
/* ActinPool (ActinPool.java:27-63), held in device memory so that a turnover cadence needs
 * no host round trip: the [actin] scalar (uM), the uM per monomer of the chamber volume
 * ((1e5^3 * 1e6) / (boxVolume_um3 * 6.022e23)) and the exact integer ledger. */
typedef struct sbx_actin_pool {
    double conc;
    double uMPerMonomer;
    int64_t totalTaken;
    int64_t totalReturned;
} sbx_actin_pool;
/* ActinPool.put (:49-52) of offsets[n] monomers, the total of a sbx_csr_scan (depoly and
 * death returns: DepolyStore.returnPoolForDepoly, DepolyStore.java:88-93) */
sbx_status sbx_actin_pool_put_total(sbx_ctx* ctx, sbx_actin_pool* pool, const int32_t* offsets, int32_t n);
/* GrowthStore.depletePoolForGrows (GrowthStore.java:94-99): ActinPool.take (:42-46) of
 * offsets[n] monomers when it is positive, the pool floored at 0 */
sbx_status sbx_actin_pool_take_total(sbx_ctx* ctx, sbx_actin_pool* pool, const int32_t* offsets, int32_t n);
/* The per-step prologue of the turnover block (FullSystemDemoHarness.java:648-651) on the
 * device: GrowthStore/DepolyStore.setCounts (step, seed, fires), AgingStore/SeverStore
 * .setFires, and GrowthStore.refreshRate (GrowthStore.java:81-91): growParams[0] =
 * (float)(onRate * conc * biochemDeltaT), 0 when fires == 0. NULL arrays are skipped. */
sbx_status sbx_turnover_begin(sbx_ctx* ctx, int32_t step, int32_t seed, int32_t fires, double onRate,
                              double biochemDeltaT, const sbx_actin_pool* pool, float* growParams,
                              int32_t* growCounts, int32_t* depolyCounts, int32_t* agingCounts,
                              int32_t* severCounts);
/* Network turnover (no reference counterpart: the reference's full demo leaves links and
 * heads attached to a dead slot): after applyDeath, every ACTIVE crosslink with an end on a
 * FREE segment becomes FREE and every head bound to a FREE segment unbinds. */
sbx_status sbx_turnover_release_dead(sbx_ctx* ctx, const int32_t* filState, int32_t nLinks, const int32_t* linkFilA,
                                     const int32_t* linkFilB, int32_t* linkState, int32_t nMotors, int32_t* boundSeg);
/* Birth holding the polymer mass constant (no reference counterpart; the request layout is
 * FilamentStore's): K = (totalReturned - totalTaken) / birthBox[3] seeds are requested,
 * request r < K at a wang-hash uniform position in the box of half-widths birthBox[0..2]
 * with a uniform in-plane axis (salts "BIR1".."BIR4"); acceptFlag[r] = r < K over reqCap. */
sbx_status sbx_birth_emit_constant_actin(sbx_ctx* ctx, int32_t reqCap, const sbx_actin_pool* pool,
                                         const float* birthBox, int32_t step, int32_t seed, int32_t* acceptFlag,
                                         float* reqCoord, float* reqUVec, float* reqYVec);
/* NodeNucleationSystem.initNewborn (NodeNucleationSystem.java:228-244): monomerCount =
 * seedParams[0], segLength = seedParams[1] in each claimed slot */
sbx_status sbx_birth_init_newborn(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                                  const int32_t* freeList, const int32_t* freeOffsets, int32_t* monomerCount,
                                  float* segLength, const float* seedParams);
/* NodeNucleationSystem.tagSeeds (:95-106): seedNode[slot] = request index (a growing tip) */
sbx_status sbx_birth_tag_seeds(sbx_ctx* ctx, int32_t K, int32_t C, const int32_t* rankOffsets,
                               const int32_t* freeList, const int32_t* freeOffsets, int32_t* seedNode);
/* pool.take(min(rankOffsets[K], freeOffsets[C]) * monomersPerBirth) (FullSystemDemoHarness.java:689-691) */
sbx_status sbx_actin_pool_take_births(sbx_ctx* ctx, sbx_actin_pool* pool, const int32_t* rankOffsets, int32_t K,
                                      const int32_t* freeOffsets, int32_t C, int32_t monomersPerBirth);
/* Turnover of packed networks (each network's filament slots a contiguous range): the
 * kernels above with the network looked up per slot or request — draws keyed by the local
 * index and the network's seed, rates from the network's table row, one pool per network —
 * and a segmented allocator (a network's slice of the global free list and request ranks
 * found at its base index). Each network gets exactly its run alone. Kernels without
 * rates, draws or allocation (apply_death, release_dead, mark_splits, recompute_drag,
 * growth_atp, filid_*, the scans) run unchanged over the packed arrays. */
typedef struct sbx_turnover_batch {
    int32_t nNet;
    const int32_t* slotKey;               /* (network, local slot) per filament slot */
    const int32_t* slotBase;              /* nNet + 1 slot offsets */
    const int32_t* seeds;                 /* nNet turnover RNG seeds */
    float* growParams;                    /* nNet x 3; [0] written by sbx_tb_begin */
    const float* depolyParams;            /* nNet x 3 */
    const float* depolyRateParams;        /* nNet x 2 */
    const float* agingParams;             /* nNet x 2 */
    const float* cofilinParams;           /* nNet x 2 */
    const float* birthBox;                /* nNet x 4 (half-widths, monomers per newborn) */
    const double* onRate;                 /* nNet growth on-rates (per uM per s) */
    sbx_actin_pool* pools;                /* nNet */
    const int32_t* birthNet;              /* network of each birth request */
    const int32_t* birthBase;             /* nNet + 1 birth-request offsets */
} sbx_turnover_batch;
sbx_status sbx_tb_begin(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t fires, double biochemDeltaT);
sbx_status sbx_tb_grow(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, const int32_t* seedNode,
                       int32_t* monomerCount, float* coord, const float* uVec, int32_t* grewFlag,
                       const int32_t* growCounts);
sbx_status sbx_tb_depoly_proxy(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, const int32_t* filState,
                               int32_t* monomerCount, float* coord, const float* uVec, const int32_t* end1NbrSlot,
                               const float* nucFrac, int32_t* returnedMon, int32_t* deathFlag,
                               const int32_t* depolyCounts);
sbx_status sbx_tb_age(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, const int32_t* filState, float* nucFrac,
                      const int32_t* agingCounts);
/* dissolve 0: cofilinAccumulate, 1: cofilinDissolve */
sbx_status sbx_tb_cofilin(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, int32_t dissolve,
                          const int32_t* filState, const float* nucFrac, float* cofFrac, const int32_t* monomerCount,
                          int32_t* severDeathFlag, int32_t* severReturnedMon, const int32_t* severCounts);
/* per network: put (take 0) or take (1) its slice total of a slot scan */
sbx_status sbx_tb_pool(sbx_ctx* ctx, const sbx_turnover_batch* tb, const int32_t* offsets, int32_t take);
sbx_status sbx_tb_split_wire(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t C, const int32_t* rankOffsets,
                             const int32_t* freeList, const int32_t* freeOffsets, int32_t* monomerCount, float* coord,
                             const float* uVec, int32_t* end1NbrSlot, int32_t* end1NbrSide, int32_t* end2NbrSlot,
                             int32_t* end2NbrSide, int32_t* seedNode, const float* splitParams);
/* space 0: requests are slots (splits), 1: birth requests; what 0 fresh cofilin, 1 fresh
 * ATP, 2 split inherit (space 0) */
sbx_status sbx_tb_formed_init(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t space, int32_t K, int32_t C,
                              const int32_t* rankOffsets, const int32_t* freeList, const int32_t* freeOffsets,
                              float* a, int32_t what);
sbx_status sbx_tb_birth_allocate(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t space, int32_t K, int32_t C,
                                 int32_t reqCap, const float* reqCoord, const float* reqUVec, const float* reqYVec,
                                 const int32_t* rankOffsets, const int32_t* freeList, const int32_t* freeOffsets,
                                 float* coord, float* uVec, float* yVec, float* brownTransScale, float* brownRotScale,
                                 int32_t* filState, const float* birthParams);
sbx_status sbx_tb_birth_emit(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t R, int32_t step, int32_t* acceptFlag,
                             float* reqCoord, float* reqUVec, float* reqYVec);
sbx_status sbx_tb_newborn(sbx_ctx* ctx, const sbx_turnover_batch* tb, int32_t R, const int32_t* rankOffsets,
                          const int32_t* freeList, const int32_t* freeOffsets, int32_t* monomerCount, float* segLength,
                          int32_t* seedNode, const float* seedParams);
sbx_status sbx_tb_pool_births(sbx_ctx* ctx, const sbx_turnover_batch* tb, const int32_t* rankOffsets,
                              const int32_t* freeOffsets, int32_t monomersPerBirth);
/* FilIDSystem.init (FilIDSystem.java:38-47): ptr = end2 neighbour (self at a chain end, -s-2 when FREE) */
sbx_status sbx_filid_init(sbx_ctx* ctx, int32_t n, const int32_t* filState, const int32_t* end2NbrSlot,
                          int32_t* ptr);
/* FilIDSystem.jump (:52-58): one pointer-doubling round, ptrOut = ptrIn[ptrIn] (ptrIn != ptrOut) */
sbx_status sbx_filid_jump(sbx_ctx* ctx, int32_t n, const int32_t* ptrIn, int32_t* ptrOut, const int32_t* filState);

/* ---------------------------------------------------------------- myosin structure
 * MotorJointSystem.joints (MotorJointSystem.java:72-197) */
sbx_status sbx_motor_joints(sbx_ctx* ctx, int32_t nB, const float* coord, const float* uVec,
                            const float* segLength, const float* bTransGam, const float* bRotGam,
                            float* forceSum, float* torqueSum, const int32_t* nucleotideState,
                            const float* jointParams);
/* DimerCouplingSystem.couple (DimerCouplingSystem.java:83-184) */
sbx_status sbx_dimer_couple(sbx_ctx* ctx, int32_t nB, const float* coord, const float* uVec,
                            const float* segLength, const float* bTransGam, const float* bRotGam,
                            float* forceSum, float* torqueSum, int32_t nD, const int32_t* motorA,
                            const int32_t* motorB, const int32_t* parallel, const float* dimerParams,
                            const int32_t* boundSeg);
/* MiniFilamentSystem.tether / backboneGather (MiniFilamentSystem.java:65-155) */
sbx_status sbx_mini_tether(sbx_ctx* ctx, int32_t nMB, const float* mCoord, const float* mUVec,
                           const float* mSegLength, const float* mBTransGam, const float* mBRotGam,
                           float* mForceSum, float* mTorqueSum, int32_t nBb, const float* bbCoord,
                           const float* bbUVec, const float* bbInvDragY, int32_t nD,
                           const int32_t* headBackboneSlot, const int32_t* motorA, const float* attachAxial,
                           float* miniData, const float* miniParams);
sbx_status sbx_mini_backbone_gather(sbx_ctx* ctx, int32_t nBb, const int32_t* bbDimerOffsets,
                                    const int32_t* bbDimerList, const float* miniData, float* bbForceSum,
                                    float* bbTorqueSum);

/* DeflectionSupport.seedAccumulators (DeflectionSupport.java:24-33): forceSum = counts[3] *
 * extForce, torqueSum = 0 (the deflection benchmark's constant load, switched by counts[3]). */
sbx_status sbx_deflection_seed_accumulators(sbx_ctx* ctx, int32_t n, float* forceSum, float* torqueSum,
                                            const float* extForce, const int32_t* counts);
/* DeflectionSupport.pinEndpoints (DeflectionSupport.java:40-58): after integration, pin p moves
 * segment pinSeg[p] so its end pinEnd[p] (1 = end1, 2 = end2) lands on pinAnchor[3p..3p+2]. */
sbx_status sbx_deflection_pin_endpoints(sbx_ctx* ctx, int32_t n, float* coord, const float* uVec,
                                        const float* segLength, int32_t nPins, const int32_t* pinSeg,
                                        const int32_t* pinEnd, const float* pinAnchor);

/* ThermostatDiag.torsionalRestore (ThermostatDiag.java:127-145): diagnostic restore of
 * every motor rod's uVec toward +z, used by the equipartition check. */
sbx_status sbx_thermostat_torsional_restore(sbx_ctx* ctx, int32_t nMotors, const float* uVec,
                                            const float* bRotGam, float* torqueSum, double coeff, double dt);

/* ================================================================ store descriptors
 * Mirrors of the reference stores (device pointers). Used by the fused step plans. */
typedef struct sbx_rigid_body {           /* RigidRodBody.java:26-84 */
    int32_t n;
    float *coord, *uVec, *yVec, *zVec, *end1, *end2, *segLength;
    float *bTransGam, *bRotGam, *bTransDiff, *bRotDiff;
    float *forceSum, *torqueSum, *randForce, *randTorque;
    float *brownTransScale, *brownRotScale;
    double *coord64;                      /* optional FP64 centres (NULL = reference FP32) */
} sbx_rigid_body;

typedef struct sbx_filament_store {       /* FilamentStore.java:29-199 */
    sbx_rigid_body body;
    int32_t *monomerCount, *end1NbrSlot, *end1NbrSide, *end2NbrSlot, *end2NbrSide, *filState;
    float *params;                        /* [0]=dt [1]=sqrt(2kT/dt) */
    float *chainParams;                   /* ChainBendingForceSystem.java:31-32 */
    int32_t *counts;                      /* [0]=n [1]=step [2]=seed [3]=loadOn */
} sbx_filament_store;

typedef struct sbx_motor_store {          /* MotorStore.java:32-161 */
    sbx_rigid_body body;                  /* 3*nMotors sub-bodies: rod, lever, head */
    int32_t nMotors;
    float *head, *uVec, *rodUVec, *reach, *bindArc;
    int32_t *boundSeg, *stats, *capStats, *cooldown;
    int32_t *nucleotideState, *forceDotPlace;
    float *forceDotFil, *forceMag, *forceDotHist;
    float *bodyParams, *jointParams, *kinParams, *nucParams;
    int32_t *counts;                      /* [0]=nMotors [1]=step [2]=seed [3]=nSeg */
    int32_t *publishParams;               /* [0]=base body-view slot */
} sbx_motor_store;

typedef struct sbx_dimer_store {          /* DimerStore.java:26-67 */
    int32_t nDimers;
    int32_t *motorA, *motorB, *parallel;
    float *dimerParams;
} sbx_dimer_store;

typedef struct sbx_minifilament_store {   /* MiniFilamentStore.java:28-135 */
    sbx_rigid_body backbone;
    int32_t nBackbones, nDimers;
    float *bbBodyParams;
    int32_t *bbCounts;                    /* [1]=step [2]=seed */
    int32_t *headBackboneSlot, *motorA;
    float *attachAxial, *miniData, *bbInvDragY, *miniParams;
    int32_t *bbDimerCount, *bbDimerOffsets, *bbDimerList;
} sbx_minifilament_store;

typedef struct sbx_crosslinker_store {    /* CrosslinkerStore.java:31-179 */
    int32_t nLinks;
    int32_t *linkFilA, *linkFilB, *linkState, *linkOrientSame, *activeLinkCount;
    float *loc1, *loc2, *xlinkData;
    float *strainHist, *torqueMagHist;
    int32_t *strainPlace, *torqueMagPlace;
    float *xlParams, *offParams, *torsionParams;
    int32_t *counts;                      /* [0]=nLinks [1]=step [2]=seed [3]=nSeg */
    /* two-pass gather CSRs (DenseContractileHarness.java:101-102) */
    int32_t *segCountA, *segOffsetsA, *segIdxA, *segCountB, *segOffsetsB, *segIdxB;
} sbx_crosslinker_store;

typedef struct sbx_grid_state {           /* SpatialBodyView.java:29-56 + SpatialGrid scratch */
    int32_t cap, totalCells;
    float *center, *boundingRadius;
    int32_t *ownerStore, *ownerSlot;
    float *gridParams, *viewParams;
    int32_t *gridDims, *gridCounts;       /* gridCounts[1] = S */
    int32_t *bodyCell, *cellCount, *chunkSum, *gridCellOffsets, *gridCellContents;
    int32_t *reachSeg, *reachCount;       /* nMotors*SBX_MAX_CAND, nMotors */
} sbx_grid_state;

/* One dense contractile network: the composition and step order of
 * DenseContractileHarness.cpuStep (DenseContractileHarness.java:350-429). */
typedef struct sbx_dense_scene {
    sbx_filament_store fil;
    sbx_motor_store mot;
    sbx_dimer_store dim;
    sbx_minifilament_store mini;
    sbx_crosslinker_store xl;
    sbx_grid_state grid;
    float *bondData, *xbParams, *boxParams;
    int32_t *segMotorCount, *segMotorOffsets, *segMotorMyo;
    int32_t seed, seedBb;                 /* SEED, SEED_BB */
    int32_t xlinkOn, xlUnbind;
} sbx_dense_scene;

typedef struct sbx_dense_plan sbx_dense_plan;

/* Builds the fused step for `scene` (pointers are kept; the scene's arrays must stay
 * alive). The fused step is bit-identical to calling the per-system entry points in
 * the DenseContractileHarness.cpuStep order. */
sbx_status sbx_dense_plan_create(sbx_ctx* ctx, const sbx_dense_scene* scene, sbx_dense_plan** out);
/* Advances steps t0, t0+1, ..., t0+nsteps-1 (the step index feeds every RNG key and
 * the containment cadence). mode 0: the call sequence of the per-system entry points
 * (zero + draws and confine + integrate + derive as the MechanicsFusion passes, which give
 * the same values); 1: one CUDA-graph replay per step of that sequence; 2: the fused persistent kernel (all nsteps in one
 * cooperative launch; available when the scene has the harness layout, see
 * sbx_dense_plan_fused_available). All three give the same bits. mode 3 (auto): the fused
 * kernel up to SBX_DENSE_AUTO_MAX_FUSED_RODS rods when available, the graph path above it,
 * where the per-system kernels' occupancy beats the persistent kernel's (measured, fused vs
 * graph ms per step: 0.070 / 0.157 at 2e4 rods, 0.092 / 0.177 at 4e4, 0.298 / 0.181 at 5e4,
 * 0.202 / 0.198 at 1e5, 1.01 / 0.44 at 5e5). */
#define SBX_DENSE_AUTO_MAX_FUSED_RODS 40960
sbx_status sbx_dense_plan_run(sbx_dense_plan* plan, int32_t t0, int32_t nsteps, int32_t mode);
/* Runs one step as the unfused per-system call sequence (reference granularity). */
sbx_status sbx_dense_step_unfused(sbx_ctx* ctx, const sbx_dense_scene* scene, int32_t t);
/* Number of kernels one fused step launches. */
int32_t sbx_dense_plan_kernels_per_step(sbx_dense_plan* plan);
/* Synchronises and reports the fused path's flags for the last run: bit0 a grid-barrier
 * wait ran out (SBX_ETIMEOUT; the state of that run is partial), bit1 a reach list
 * exceeded SBX_MAX_CAND (SBX_EOVERFLOW; counts continue past the cap, as the reference),
 * bit2 a bulk-copy wait ran out (SBX_ETIMEOUT), bit3 a linked-list walk ran past its bound
 * (SBX_ESTATE). */
sbx_status sbx_dense_plan_status(sbx_dense_plan* plan, int32_t* flags);
/* 1 when the fused persistent path is available for this scene (else mode 2 returns SBX_ESTATE) */
int32_t sbx_dense_plan_fused_available(sbx_dense_plan* plan);
/* Re-reads the chain topology for the fused path after the scene's filament topology changed
 * (a turnover cadence: growth splits, deaths, births into FREE slots): rod groups, whether
 * neighbours cross groups, joint sharing. Synchronises the plan's stream. The graph and
 * per-system paths need no refresh. */
sbx_status sbx_dense_plan_refresh(sbx_dense_plan* plan);
/* cooperative grid size (CTAs) of the fused path */
int32_t sbx_dense_plan_fused_grid(sbx_dense_plan* plan);
/* Phase timing of the fused path: when dev_times (device int64 array of
 * nsteps*SBX_FUSED_PHASES) is set, each run writes the %globaltimer value (ns) after every
 * phase barrier of every step; NULL switches it off. */
#define SBX_FUSED_PHASES 7
sbx_status sbx_dense_plan_phase_times(sbx_dense_plan* plan, int64_t* dev_times);
/* Test hook for failure detection: the fused kernel's grid barrier waits for `extra`
 * arrivals that never come, so its bounded wait runs out and the run reports
 * SBX_ETIMEOUT. 0 restores normal operation. */
sbx_status sbx_dense_plan_test_barrier_extra(sbx_dense_plan* plan, int32_t extra);
/* Supplied-noise mode of the dense step: both the library and a CPU implementation of the
 * step consume the same Gaussian array. Each step t in [t0, t0 + nsteps) takes its six
 * Gaussians per body from planar device arrays fil[t - t0][6][nRods],
 * mot[t - t0][6][3 nMotors] and bb[t - t0][6][nBackbones] (gfx gfy gfz gtx gty gtz, the
 * order of the Box-Muller outputs of BrownianForceSystem.brownianForce,
 * BrownianForceSystem.java:78-92) instead of the Wang-hash draws; the amplitudes, the rest
 * of the step and every other RNG stream (release, nucleotide cycle, Bell unbind) are
 * unchanged. NULL switches the mode off. The arrays must stay alive while the mode is on;
 * they are checked for NaN/Inf here (SBX_ENONFINITE, mode left unchanged). A run whose steps
 * leave [t0, t0 + nsteps) returns SBX_EINVAL. Not available for packed plans. All paths
 * (per-system, graph, fused) honour it and give the same bits. */
typedef struct sbx_dense_noise {
    const float *fil, *mot, *bb;
    int32_t t0, nsteps;
} sbx_dense_noise;
sbx_status sbx_dense_plan_set_noise(sbx_dense_plan* plan, const sbx_dense_noise* noise);
/* Counters of the fused kernel's capacity fallbacks since the plan was created (or since
 * the last call with reset != 0), for tests that must show the fallback paths ran:
 * out[0] grid cells with more than the fixed row slots (overflow list walked),
 * out[1] segments with more link ends than the fixed slots, out[2] segments with more bound
 * motors than the fixed slots, out[3] link payload entries read from global memory past
 * the rod CTA's staging capacity, out[4] motor reactions read from global memory past the
 * staged ones, out[5] motor rows longer than the sorted-slot capacity (repeated-minimum
 * walk), out[6] reach lists longer than SBX_MAX_CAND, out[7] reserved; `out` holds
 * SBX_FUSED_STATS values. */
#define SBX_FUSED_STATS 8
sbx_status sbx_dense_plan_fused_stats(sbx_dense_plan* plan, int64_t* out, int32_t reset);
/* Test hook: lowers the fused kernel's capacities (link payload entries a rod CTA stages,
 * motor reactions staged per segment, motor slots sorted per segment, fixed row slots per
 * segment row (link rows and motor rows alike), fixed slots per grid cell) to exercise the fallback paths on ordinary
 * scenes; each value is clamped to [0, the compiled capacity], a negative value restores
 * the compiled capacity. Takes effect at the next run; the results are the same bits. */
sbx_status sbx_dense_plan_test_caps(sbx_dense_plan* plan, int32_t entCap, int32_t motorCap, int32_t motorIds,
                                    int32_t rowSlots, int32_t cellSlots);
/* Waits for the device and frees the plan; safe after the plan's context was destroyed. */
sbx_status sbx_dense_plan_destroy(sbx_dense_plan* plan);

/* ---------------------------------------------------------------- batched networks
 * Many independent dense networks packed into one sbx_dense_scene: network k owns a
 * contiguous index range of every store (cross-store indices offset accordingly) and its
 * own grid cells. The step runs one launch per phase for all networks; the draws are keyed
 * by each item's local index and its network's seed, the grid and walls are the
 * network's own, so each network's result equals its run alone, bit for bit.
 * Key arrays hold (network, local index) int32 pairs per item. */
typedef struct sbx_batch {
    int32_t nNet;
    int32_t *segKey, *motKey, *bbKey, *linkKey;
    int32_t *seeds;                       /* nNet x 3: SEED (motors, links), SEED_BB, filament counts[2] */
    float *gridParams;                    /* nNet x 6: each network's gridParams */
    int32_t *gridDims;                    /* nNet x 4: nX, nY, nZ, first global cell */
    float *boxParams;                     /* nNet x 8: each network's boxParams */
} sbx_batch;
/* the batched forms of the step's network-dependent kernels (same arithmetic as the
 * single-network entry points; perKey = 3 for motor bodies, keyed by their motor) */
sbx_status sbx_brownian_force_batched(sbx_ctx* ctx, int32_t n, int32_t perKey, float* rF, float* rT, const float* bTG,
                                      const float* bRG, const float* tSc, const float* rSc, const float* params,
                                      const int32_t* counts, const int32_t* key, const int32_t* seeds,
                                      int32_t seedCol);
sbx_status sbx_nucleotide_release_batched(sbx_ctx* ctx, int32_t nM, int32_t* boundSeg, const float* fdf,
                                          const float* fm, int32_t* cooldown, int32_t* stats, int32_t* capStats,
                                          const float* kp, const int32_t* counts, const int32_t* motKey,
                                          const int32_t* seeds);
sbx_status sbx_nucleotide_cycle_batched(sbx_ctx* ctx, int32_t nM, int32_t* state, const int32_t* boundSeg,
                                        const float* hist, const float* np, const int32_t* counts,
                                        const int32_t* motKey, const int32_t* seeds);
sbx_status sbx_xlink_unbind_batched(sbx_ctx* ctx, int32_t nSeg, const float* fU, const float* fE1, int32_t nLinks,
                                    const int32_t* A, const int32_t* B, const float* loc1, const float* loc2,
                                    int32_t* state, float* hist, int32_t* place, const float* op,
                                    const int32_t* counts, const int32_t* linkKey, const int32_t* seeds);
sbx_status sbx_grid_body_cell_batched(sbx_ctx* ctx, int32_t cap, const float* center, const int32_t* counts,
                                      int32_t* bodyCell, int32_t nSeg, const int32_t* segKey, const int32_t* motKey,
                                      const float* gpTab, const int32_t* gdTab);
sbx_status sbx_binding_grid_reachable_batched(sbx_ctx* ctx, const float* head, const float* uVec,
                                              const float* rodUVec, int32_t nSeg, const float* e1, const float* e2,
                                              const int32_t* offsets, const int32_t* contents,
                                              const int32_t* ownerStore, const int32_t* ownerSlot, int32_t* reachSeg,
                                              int32_t* reachCount, const float* kp, int32_t nM,
                                              const int32_t* motKey, const float* gpTab, const int32_t* gdTab);
sbx_status sbx_fusion_grid_reachable_batched(sbx_ctx* ctx, const float* head, const float* uVec,
                                             const float* rodUVec, const int32_t* offsets, const float* cellEnd1,
                                             const float* cellEnd2, int32_t* reachSeg, int32_t* reachCount,
                                             const float* kp, int32_t nM, const int32_t* motKey,
                                             const float* gpTab, const int32_t* gdTab);
sbx_status sbx_confine_batched(sbx_ctx* ctx, int32_t n, const float* coord, const float* uVec,
                               const float* segLength, const float* bTG, float* F, float* T, const float* boxTab,
                               const int32_t* counts, const int32_t* key);
/* ---------------------------------------------------------------- observables
 * Per network k of a single or packed scene (segBase/linkBase/motBase: nNet+1 device
 * offsets of the network's index ranges). Deterministic FP64 reductions: one block per
 * network, thread t sums items t, t+256, ... in index order, then a fixed tree.
 * RMS extent of the ACTIVE filament rods about their mean (FullSystemDemoHarness.filRms,
 * FullSystemDemoHarness.java:1047-1055): out[2k] = R_rms (um), out[2k+1] = rods counted.
 * coord64 (FP64 centres) is used when given; filState may be NULL (all ACTIVE). */
sbx_status sbx_obs_extent(sbx_ctx* ctx, int32_t nNet, const int32_t* segBase, int32_t nSeg, const float* coord,
                          const double* coord64, const int32_t* filState, double* out);
/* Mean in-plane network stress: out[k] = -(1/(2V_k)) sum (r_x F_x + r_y F_y) over ACTIVE
 * crosslinks (r = attachment A - attachment B, F = the payload force on A) and bound heads
 * (r = head tip - attachment point, F = the payload force on the head), r in m, V in um^3
 * (volume[k]), Pa; positive = tension. linkBase or motBase may be NULL to leave a term out. */
sbx_status sbx_obs_stress(sbx_ctx* ctx, int32_t nNet, int32_t nSeg, const float* coord, const float* uVec,
                          const float* end1, const float* segLength, const int32_t* linkBase, const int32_t* linkFilA,
                          const int32_t* linkFilB, const int32_t* linkState, const float* loc1, const float* loc2,
                          const float* xlinkData, int32_t nMotors, const int32_t* motBase, const float* motCoord,
                          const float* motUVec, const int32_t* boundSeg, const float* bindArc,
                          const float* bondData, double headLen, const float* volume, double* out);
/* Largest cluster: components over ACTIVE segments and backbones joined by chain links,
 * ACTIVE crosslinks and bound heads (segment -- its head's backbone, motorBackbone[m]).
 * `rounds` hook-and-compress rounds (each skipped once the previous one changed nothing);
 * flags[rounds] scratch, flags[rounds-1] != 0 afterwards means not converged. label
 * receives each node's component id (its smallest node id; -1 for FREE segments), size the
 * component sizes in segments; out[2k] = largest component (segments), out[2k+1] = ACTIVE
 * segments of network k. */
sbx_status sbx_obs_clusters(sbx_ctx* ctx, int32_t nNet, const int32_t* segBase, int32_t nSeg, const int32_t* filState,
                            const int32_t* end2NbrSlot, int32_t nLinks, const int32_t* linkFilA,
                            const int32_t* linkFilB, const int32_t* linkState, int32_t nMotors,
                            const int32_t* boundSeg, const int32_t* motorBackbone, int32_t nBackbones,
                            int32_t rounds, int32_t* label, int32_t* size, int32_t* flags, int32_t* out);
/* ---------------------------------------------------------------- surrogate (MLP ensemble)
 * C[M x N] = A[M x K] . B[N x K]^T on the tensor cores (tcgen05, BF16 operands, FP32
 * accumulation), K <= 256, for nz independent problems (ensemble members) at the given
 * element strides. A and B are row-major BF16 (uint16 bit patterns). Epilogue per element:
 * v = acc (+ bias[n]); outF = v (FP32, optional); a = act ? GELU(v) : v (act 1 = exact GELU);
 * out = bf16(a) row-major (optional) and outT = bf16(a) transposed, N x M with leading
 * dimension ldt (optional). errFlag (optional device int) gets bit 0 when an MMA completion
 * wait ran out. */
sbx_status sbx_mlp_gemm_bf16(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t N, int32_t K, const void* A, int32_t lda,
                             int64_t strideA, const void* B, int32_t ldb, int64_t strideB, const float* bias,
                             int64_t strideBias, int32_t act, void* out, int32_t ldo, int64_t strideOut, void* outT,
                             int32_t ldt, int64_t strideOutT, float* outF, int32_t ldf, int64_t strideOutF,
                             int32_t* errFlag);
/* g = dA * GELU'(Z) (Z NULL: g = dA) as BF16, row-major M x N and transposed N x M */
sbx_status sbx_mlp_gelu_backward(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t N, const float* dA, const float* Z,
                                 int64_t strideMN, void* g, void* gT, int64_t strideG, int64_t strideGT);
/* out[n] = sum over rows of a BF16 M x N matrix, rows in order (bias gradients) */
sbx_status sbx_mlp_colsum_bf16(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t N, const void* in, int64_t strideIn,
                               float* out, int64_t strideOut);
/* mean-squared-error gradient over the first nOut of Np columns (0 on the padding); loss
 * (optional, nz floats) accumulates the mean squared error */
sbx_status sbx_mlp_mse_grad(sbx_ctx* ctx, int32_t nz, int32_t M, int32_t Np, int32_t nOut, const float* y,
                            int64_t strideY, const float* t, int64_t strideT, float* g, int64_t strideG, float* loss);
/* Adam step (bias-corrected with stepNumber) on FP32 master weights N x K; refreshes the
 * BF16 copy (N x K) and, when given, its transpose (K x N) */
sbx_status sbx_mlp_adam(sbx_ctx* ctx, int32_t nz, int32_t N, int32_t K, float* w, const float* gw, float* m, float* v,
                        int64_t stride, float lr, float beta1, float beta2, float eps, int32_t stepNumber,
                        void* wBf16, void* wBf16T, int64_t strideB, int64_t strideBT);
/* A plan over a packed scene (graph and per-system paths; the fused kernel is for one
 * network). `batch` is copied; its arrays must stay alive. */
sbx_status sbx_dense_plan_create_batched(sbx_ctx* ctx, const sbx_dense_scene* scene, const sbx_batch* batch,
                                         sbx_dense_plan** out);

/* Free rods (DiffusionHarness cpuStepFdt order: brownian -> integrate -> derive).
 * Runs nsteps steps (t0..) in one persistent launch that keeps each rod in registers.
 * noise_mode 0 = Wang hash (reference), 1 = Philox (philox_seed), 2 = supplied
 * (noise = planar [nsteps][6][n]). */
sbx_status sbx_free_rods_run(sbx_ctx* ctx, sbx_filament_store* fil, int32_t t0, int32_t nsteps,
                             int32_t noise_mode, uint64_t philox_seed, const float* noise);

#ifdef __cplusplus
}
#endif
#endif /* SOFTBOX_B200_H */
