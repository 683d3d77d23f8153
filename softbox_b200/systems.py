"""The reference's System classes, re-exposed over the B200 library.

Class and method names, argument order and argument meaning follow the Java static
methods (package softbox/ of the reference), with torch CUDA tensors in place of
TornadoVM FloatArray / IntArray buffers. Lengths are taken from the tensors exactly as
the Java code reads them with getSize(). Every method launches on the default library
context (torch's current stream on cuda:0); errors raise runtime.SbxError. There is no
CPU path.
"""
from .runtime import default_context


def _ctx():
    return default_context()


def _n3(a):
    return a.numel() // 3


class DragTensorSystem:                      # DragTensorSystem.java
    @staticmethod
    def run_filament(monomerCount, end1NbrSlot, end2NbrSlot, aeta, segLength, bTransGam, bRotGam, bTransDiff,
                     bRotDiff):
        _ctx()("sbx_drag_run_filament", segLength.numel(), monomerCount, end1NbrSlot, end2NbrSlot, float(aeta),
               segLength, bTransGam, bRotGam, bTransDiff, bRotDiff)

    @staticmethod
    def run_motor(nMotors, aeta, segLength, bTransGam, bRotGam, bTransDiff, bRotDiff):
        _ctx()("sbx_drag_run_motor", nMotors, float(aeta), segLength, bTransGam, bRotGam, bTransDiff, bRotDiff)

    @staticmethod
    def run_backbone(bbLen, aeta, segLength, bTransGam, bRotGam, bTransDiff, bRotDiff, bbInvDragY):
        _ctx()("sbx_drag_run_backbone", segLength.numel(), float(bbLen), float(aeta), segLength, bTransGam, bRotGam,
               bTransDiff, bRotDiff, bbInvDragY)


class BrownianForceSystem:                   # BrownianForceSystem.java:44
    @staticmethod
    def brownianForce(randForce, randTorque, bTransGam, bRotGam, brownTransScale, brownRotScale, params, counts):
        _ctx()("sbx_brownian_force", _n3(randForce), randForce, randTorque, bTransGam, bRotGam, brownTransScale,
               brownRotScale, params, counts)

    @staticmethod
    def brownianForcePhilox(randForce, randTorque, bTransGam, bRotGam, brownTransScale, brownRotScale, params,
                            counts, seed):
        _ctx()("sbx_brownian_force_philox", _n3(randForce), randForce, randTorque, bTransGam, bRotGam,
               brownTransScale, brownRotScale, params, counts, int(seed))

    @staticmethod
    def brownianForceSupplied(randForce, randTorque, bTransGam, bRotGam, brownTransScale, brownRotScale, params,
                              noise):
        _ctx()("sbx_brownian_force_supplied", _n3(randForce), randForce, randTorque, bTransGam, bRotGam,
               brownTransScale, brownRotScale, params, noise)


class RigidRodLangevinIntegrationSystem:     # RigidRodLangevinIntegrationSystem.java:33
    @staticmethod
    def integrate(coord, uVec, yVec, forceSum, torqueSum, randForce, randTorque, bTransGam, bRotGam, params,
                  counts=None, coord64=None):
        _ctx()("sbx_integrate", _n3(coord), coord, coord64, uVec, yVec, forceSum, torqueSum, randForce, randTorque,
               bTransGam, bRotGam, params)


class DerivedGeometrySystem:                 # DerivedGeometrySystem.java:27
    @staticmethod
    def derive(coord, uVec, yVec, zVec, end1, end2, segLength, counts=None):
        _ctx()("sbx_derive", _n3(coord), coord, uVec, yVec, zVec, end1, end2, segLength)


class ContainmentSystem:                     # ContainmentSystem.java:58
    @staticmethod
    def confine(coord, uVec, segLength, bTransGam, forceSum, torqueSum, boxParams, counts):
        _ctx()("sbx_confine", _n3(coord), coord, uVec, segLength, bTransGam, forceSum, torqueSum, boxParams, counts)


class MechanicsFusion:                       # MechanicsFusion.java:52-338
    @staticmethod
    def forceBuild(forceSum, torqueSum, randForce, randTorque, bTransGam, bRotGam, brownTransScale, brownRotScale,
                   params, counts):
        _ctx()("sbx_fusion_force_build", _n3(forceSum), forceSum, torqueSum, randForce, randTorque, bTransGam,
               bRotGam, brownTransScale, brownRotScale, params, counts)

    @staticmethod
    def integDerive(coord, uVec, yVec, zVec, segLength, end1, end2, forceSum, torqueSum, randForce, randTorque,
                    bTransGam, bRotGam, params, coord64=None):
        _ctx()("sbx_fusion_integ_derive", _n3(coord), coord, coord64, uVec, yVec, zVec, segLength, end1, end2,
               forceSum, torqueSum, randForce, randTorque, bTransGam, bRotGam, params)

    @staticmethod
    def integDeriveConfined(coord, uVec, yVec, zVec, segLength, end1, end2, forceSum, torqueSum, randForce,
                            randTorque, bTransGam, bRotGam, boxParams, counts, coord64=None):
        _ctx()("sbx_fusion_integ_derive_confined", _n3(coord), coord, coord64, uVec, yVec, zVec, segLength, end1,
               end2, forceSum, torqueSum, randForce, randTorque, bTransGam, bRotGam, boxParams, counts)


class ChainBendingForceSystem:               # ChainBendingForceSystem.java
    @staticmethod
    def zeroAccumulators(forceSum, torqueSum, counts=None):
        _ctx()("sbx_zero_accumulators", _n3(forceSum), forceSum, torqueSum)

    @staticmethod
    def chainForces(coord, uVec, segLength, end2NbrSlot, end2NbrSide, end1NbrSlot, end1NbrSide, bTransGam, bRotGam,
                    forceSum, torqueSum, chainParams, counts=None):
        _ctx()("sbx_chain_forces", _n3(coord), coord, uVec, segLength, end2NbrSlot, end2NbrSide, end1NbrSlot,
               end1NbrSide, bTransGam, bRotGam, forceSum, torqueSum, chainParams)


class FilamentStore:                         # FilamentStore.java:275-328
    @staticmethod
    def publishToBodyView(coord, segLength, center, boundingRadius, ownerStore, ownerSlot, viewParams, counts=None,
                          filState=None):
        _ctx()("sbx_filament_publish", _n3(coord), coord, segLength, _n3(center), center, boundingRadius,
               ownerStore, ownerSlot, viewParams, filState)


class MotorStore:                            # MotorStore.java:300-347
    @staticmethod
    def publishHeadFromBody(bodyCoord, bodyUVec, bodySegLength, head, uVec, rodUVec, counts=None):
        _ctx()("sbx_motor_publish_head", _n3(head), bodyCoord, bodyUVec, bodySegLength, head, uVec, rodUVec)

    @staticmethod
    def publishToBodyView(head, reach, center, boundingRadius, ownerStore, ownerSlot, publishParams, counts=None):
        _ctx()("sbx_motor_publish", _n3(head), head, reach, _n3(center), center, boundingRadius, ownerStore, ownerSlot,
               publishParams)


class SpatialGrid:                           # SpatialGrid.java
    MAX_CAND = 256
    GRID_SCAN_CHUNK = 512

    @staticmethod
    def bodyCell(center, gridParams, gridDims, counts, bodyCell):
        _ctx()("sbx_grid_body_cell", _n3(center), center, gridParams, gridDims, counts, bodyCell)

    @staticmethod
    def build(bodyCell, counts, gridDims, cellCount, chunkSum, gridCellOffsets, gridCellContents):
        """gridZero + gridHistogram + gridScanLocal/Chunks/Add + gridScatter in one call."""
        _ctx()("sbx_grid_build", bodyCell.numel(), bodyCell, counts, cellCount.numel(), cellCount, chunkSum,
               gridCellOffsets, gridCellContents, gridCellContents.numel())

    @staticmethod
    def broadPhase(center, boundingRadius, bodyCell, gridCellOffsets, gridCellContents, gridDims, gridParams, counts,
                   candPartner, candCount):
        _ctx()("sbx_grid_broad_phase", _n3(center), center, boundingRadius, bodyCell, gridCellOffsets,
               gridCellContents, gridDims, gridParams, counts, candPartner, candCount)

    @staticmethod
    def bruteForce(center, boundingRadius, gridParams, counts, brutePartner, bruteCount):
        _ctx()("sbx_grid_brute_force", _n3(center), center, boundingRadius, gridParams, counts, brutePartner,
               bruteCount)


class BindingDetectionSystem:                # BindingDetectionSystem.java
    @staticmethod
    def gridReachable(head, uVec, rodUVec, segEnd1, segEnd2, gridParams, gridDims, gridCellOffsets,
                      gridCellContents, ownerStore, ownerSlot, motorReachSeg, motorReachCount, kinParams, counts=None):
        _ctx()("sbx_binding_grid_reachable", head, uVec, rodUVec, _n3(segEnd1), segEnd1, segEnd2, gridParams,
               gridDims, gridCellOffsets, gridCellContents, ownerStore, ownerSlot, motorReachSeg, motorReachCount,
               kinParams, _n3(head))

    @staticmethod
    def bruteReachable(head, uVec, rodUVec, segEnd1, segEnd2, bruteReachSeg, bruteReachCount, kinParams,
                       counts=None):
        _ctx()("sbx_binding_brute_reachable", head, uVec, rodUVec, _n3(segEnd1), segEnd1, segEnd2, bruteReachSeg,
               bruteReachCount, kinParams, _n3(head))

    @staticmethod
    def bindNearest(head, uVec, rodUVec, segEnd1, segEnd2, motorCandSeg, motorCandCount, boundSeg, bindArc,
                    kinParams, counts=None):
        _ctx()("sbx_binding_bind_nearest", head, uVec, rodUVec, _n3(segEnd1), segEnd1, segEnd2, motorCandSeg,
               motorCandCount, boundSeg, bindArc, kinParams, _n3(head))


class NucleotideCycleSystem:                 # NucleotideCycleSystem.java
    @staticmethod
    def cycle(nucleotideState, boundSeg, forceDotHist, nucParams, counts):
        _ctx()("sbx_nucleotide_cycle", nucleotideState.numel(), nucleotideState, boundSeg, forceDotHist, nucParams,
               counts)

    @staticmethod
    def catchSlipRelease(boundSeg, forceDotFil, forceMag, cooldown, stats, capStats, kinParams, counts):
        _ctx()("sbx_nucleotide_release", boundSeg.numel(), boundSeg, forceDotFil, forceMag, cooldown, stats,
               capStats, kinParams, counts)


class CrossBridgeSystem:                     # CrossBridgeSystem.java
    STRIDE = 13

    @staticmethod
    def bondForces(motorCoord, motorUVec, motorYVec, motorBRotGam, filCoord, filUVec, filYVec, filBRotGam,
                   filSegLength, boundSeg, bindArc, nucleotideState, bondData, xbParams):
        _ctx()("sbx_xbridge_bond_forces", _n3(motorCoord), motorCoord, motorUVec, motorYVec, motorBRotGam,
               _n3(filCoord), filCoord, filUVec, filYVec, filBRotGam, filSegLength, boundSeg, bindArc,
               nucleotideState, bondData, xbParams)

    @staticmethod
    def applyHeadForce(bondData, bodyForceSum, bodyTorqueSum, counts=None):
        _ctx()("sbx_xbridge_apply_head_force", _n3(bodyForceSum), bondData, bodyForceSum, bodyTorqueSum)

    @staticmethod
    def registerForceDot(bondData, boundSeg, forceDotFil, forceMag, forceDotHist, forceDotPlace, counts=None):
        _ctx()("sbx_xbridge_register_force_dot", boundSeg.numel(), bondData, boundSeg, forceDotFil, forceMag,
               forceDotHist, forceDotPlace)

    @staticmethod
    def csrScan(counts, segMotorCount, segMotorOffsets):
        """CrossBridgeSystem.csrScan (CrossBridgeSystem.java:198-205): n = counts[3] rows (host value)."""
        n = int(counts[3]) if not hasattr(counts, "device") or counts.device.type == "cpu" else int(counts[3].item())
        _ctx()("sbx_csr_scan", n, segMotorCount, segMotorOffsets)

    @staticmethod
    def csrBuild(keys, nRows, rowCount, rowOffsets, rowList):
        """csrHistogram + csrScan + csrScatter (and the csrChunk* variant) in one call."""
        _ctx()("sbx_csr_build", keys, keys.numel(), int(nRows), rowCount, rowOffsets, rowList)

    @staticmethod
    def segGather(segMotorOffsets, segMotorMyo, bondData, filForceSum, filTorqueSum, counts=None):
        _ctx()("sbx_xbridge_seg_gather", segMotorOffsets.numel() - 1, segMotorOffsets, segMotorMyo, bondData,
               filForceSum, filTorqueSum)

    @staticmethod
    def bruteGather(boundSeg, bondData, bForceSum, bTorqueSum, counts=None):
        _ctx()("sbx_xbridge_brute_gather", _n3(bForceSum), boundSeg.numel(), boundSeg, bondData, bForceSum,
               bTorqueSum)


class CrosslinkerSystem:                     # CrosslinkerSystem.java
    @staticmethod
    def countActiveLinks(linkState, linkFilA, linkFilB, activeLinkCount, formCounts=None):
        _ctx()("sbx_xlink_count_active", linkState.numel(), linkState, linkFilA, linkFilB, activeLinkCount.numel(),
               activeLinkCount)

    @staticmethod
    def linkForces(filCoord, filUVec, filEnd1, filBTransGam, linkFilA, linkFilB, loc1, loc2, filLinkCt, xlinkData,
                   xlParams):
        _ctx()("sbx_xlink_forces", _n3(filCoord), filCoord, filUVec, filEnd1, filBTransGam, linkFilA.numel(),
               linkFilA, linkFilB, loc1, loc2, filLinkCt, xlinkData, xlParams)

    @staticmethod
    def linkTorsion(filUVec, linkFilA, linkFilB, linkState, linkOrientSame, torqueMagHist, torqueMagPlace,
                    xlinkData, torsionParams):
        _ctx()("sbx_xlink_torsion", _n3(filUVec), filUVec, linkFilA.numel(), linkFilA, linkFilB, linkState,
               linkOrientSame, torqueMagHist, torqueMagPlace, xlinkData, torsionParams)

    @staticmethod
    def segGatherA(segOffsets, segLinkIdx, xlinkData, linkState, filForceSum, filTorqueSum, counts=None):
        _ctx()("sbx_xlink_seg_gather", 0, segOffsets.numel() - 1, segOffsets, segLinkIdx, xlinkData, linkState,
               filForceSum, filTorqueSum)

    @staticmethod
    def segGatherB(segOffsets, segLinkIdx, xlinkData, linkState, filForceSum, filTorqueSum, counts=None):
        _ctx()("sbx_xlink_seg_gather", 1, segOffsets.numel() - 1, segOffsets, segLinkIdx, xlinkData, linkState,
               filForceSum, filTorqueSum)

    @staticmethod
    def bruteGather(linkFilA, linkFilB, xlinkData, linkState, bForceSum, bTorqueSum, counts=None):
        _ctx()("sbx_xlink_brute_gather", _n3(bForceSum), linkFilA.numel(), linkFilA, linkFilB, xlinkData, linkState,
               bForceSum, bTorqueSum)

    @staticmethod
    def unbind(filCoord, filUVec, filEnd1, linkFilA, linkFilB, loc1, loc2, linkState, strainHist, strainPlace,
               offParams, counts):
        _ctx()("sbx_xlink_unbind", _n3(filCoord), filUVec, filEnd1, linkFilA.numel(), linkFilA, linkFilB, loc1, loc2,
               linkState, strainHist, strainPlace, offParams, counts)

    # ---- formation (CrosslinkerSystem.java:405-756) and the free-list allocator (:297-345)
    FORM_MAXC = 256

    @staticmethod
    def filFilCandidates(filCoord, filSegLength, filID, reqFilA, reqFilB, formParams, formCounts):
        _ctx()("sbx_xlink_fil_fil_candidates", _n3(filCoord), filCoord, filSegLength, filID, reqFilA.numel(),
               reqFilA, reqFilB, formParams, formCounts)

    @staticmethod
    def gridFormCount(filCoord, filSegLength, filID, gridParams, gridDims, gridCellOffsets, gridCellContents,
                      candCountSeg, formParams, formCounts=None):
        _ctx()("sbx_xlink_grid_form_count", _n3(filCoord), filCoord, filSegLength, filID, gridParams, gridDims,
               gridCellOffsets, gridCellContents, candCountSeg, formParams)

    @staticmethod
    def gridFormScan(candCountSeg, candBaseSeg, reqFilA, reqFilB, formCounts):
        _ctx()("sbx_xlink_grid_form_scan", candCountSeg.numel(), candCountSeg, candBaseSeg, reqFilA.numel(), reqFilA,
               reqFilB, formCounts)

    @staticmethod
    def gridFormEmit(filCoord, filSegLength, filID, gridParams, gridDims, gridCellOffsets, gridCellContents,
                     candBaseSeg, candCountSeg, reqFilA, reqFilB, formParams, formCounts=None):
        _ctx()("sbx_xlink_grid_form_emit", _n3(filCoord), filCoord, filSegLength, filID, gridParams, gridDims,
               gridCellOffsets, gridCellContents, candBaseSeg, candCountSeg, reqFilA.numel(), reqFilA, reqFilB,
               formParams)

    @staticmethod
    def formGates(filUVec, filEnd1, filEnd2, filSegLength, reqFilA, reqFilB, reqLoc1, reqLoc2, reqOrient, gatePass,
                  formParams, formCounts):
        _ctx()("sbx_xlink_form_gates", _n3(filUVec), filUVec, filEnd1, filEnd2, filSegLength, reqFilA.numel(),
               reqFilA, reqFilB, reqLoc1, reqLoc2, reqOrient, gatePass, formParams, formCounts)

    @staticmethod
    def formAdmitReduce(reqFilA, reqFilB, gatePass, minCand, formCounts=None):
        _ctx()("sbx_xlink_form_admit_reduce", reqFilA.numel(), reqFilA, reqFilB, gatePass, minCand.numel(), minCand)

    @staticmethod
    def formAdmit(reqFilA, reqFilB, reqLoc1, reqLoc2, gatePass, minCand, activeLinkCount, linkState, linkFilA,
                  linkFilB, loc1, loc2, acceptFlag, formParams, formCounts=None):
        _ctx()("sbx_xlink_form_admit", reqFilA.numel(), reqFilA, reqFilB, reqLoc1, reqLoc2, gatePass, minCand,
               activeLinkCount, linkState.numel(), linkState, linkFilA, linkFilB, loc1, loc2, acceptFlag, formParams)

    @staticmethod
    def freeFlags(linkState, freeCount, allocCounts=None):
        _ctx()("sbx_xlink_free_flags", freeCount.numel(), linkState, freeCount)

    @staticmethod
    def freeScatter(linkState, freeOffsets, freeList, allocCounts=None):
        _ctx()("sbx_xlink_free_scatter", freeList.numel(), linkState, freeOffsets, freeList)

    @staticmethod
    def allocate(reqFilA, reqFilB, reqLoc1, reqLoc2, rankOffsets, freeList, freeOffsets, linkFilA, linkFilB, loc1,
                 loc2, linkState, strainHist, strainPlace, allocCounts=None, K=None):
        K = reqFilA.numel() if K is None else K
        _ctx()("sbx_xlink_allocate", K, reqFilA, reqFilB, reqLoc1, reqLoc2, rankOffsets, freeList, freeOffsets,
               freeList.numel(), linkFilA, linkFilB, loc1, loc2, linkState, strainHist, strainPlace)

    @staticmethod
    def placeOrient(reqOrient, rankOffsets, freeList, freeOffsets, linkOrientSame, torqueMagHist, torqueMagPlace,
                    allocCounts=None, K=None):
        K = reqOrient.numel() if K is None else K
        _ctx()("sbx_xlink_place_orient", K, reqOrient, rankOffsets, freeList, freeOffsets, freeList.numel(),
               linkOrientSame, torqueMagHist, torqueMagPlace)


class FormationGrid:                         # FormationGrid.java:28-109
    """The dedicated crosslinker-formation grid: one body per segment, cell size
    >= max segment length + grab so the 27-cell stencil is complete."""

    def __init__(self, n_seg, gx, gy, gz, cell_size, grab, actin_radius, device="cuda"):
        import math
        import torch
        i32 = dict(dtype=torch.int32, device=device)
        f32 = dict(dtype=torch.float32, device=device)
        self.nSeg = n_seg
        nX = 1 + int(math.ceil(2 * gx / cell_size))
        nY = 1 + int(math.ceil(2 * gy / cell_size))
        nZ = 1 + int(math.ceil(2 * gz / cell_size))
        self.totalCells = nX * nY * nZ
        self.viewParams = torch.tensor([actin_radius], **f32)
        self.gridParams = torch.tensor([-gx, -gy, -gz, cell_size, 1.0 / cell_size, grab], **f32)
        self.gridDims = torch.tensor([nX, nY, nZ, self.totalCells], **i32)
        self.gridCounts = torch.tensor([0, n_seg, 0, 0], **i32)
        self.center = torch.zeros(3 * n_seg, **f32)
        self.boundingRadius = torch.zeros(n_seg, **f32)
        self.ownerStore = torch.zeros(n_seg, **i32)
        self.ownerSlot = torch.zeros(n_seg, **i32)
        self.bodyCell = torch.full((n_seg,), -1, **i32)
        self.cellCount = torch.zeros(self.totalCells, **i32)
        self.chunkSum = torch.zeros((self.totalCells + 511) // 512 + 1, **i32)
        self.gridCellOffsets = torch.zeros(self.totalCells + 1, **i32)
        self.gridCellContents = torch.full((n_seg,), -1, **i32)
        self.candCountSeg = torch.zeros(n_seg, **i32)
        self.candBaseSeg = torch.zeros(n_seg + 1, **i32)

    def build(self, filCoord, filSegLength, filState=None):
        """publishToBodyView -> bodyCell -> counting sort (FormationGrid.buildCpu)."""
        c = _ctx()
        c("sbx_filament_publish", self.nSeg, filCoord, filSegLength, self.nSeg, self.center, self.boundingRadius,
          self.ownerStore, self.ownerSlot, self.viewParams, filState)
        SpatialGrid.bodyCell(self.center, self.gridParams, self.gridDims, self.gridCounts, self.bodyCell)
        SpatialGrid.build(self.bodyCell, self.gridCounts, self.gridDims, self.cellCount, self.chunkSum,
                          self.gridCellOffsets, self.gridCellContents)

    def formCandidates(self, filCoord, filSegLength, filID, reqFilA, reqFilB, formParams, formCounts):
        """gridFormCount -> gridFormScan -> gridFormEmit (FormationGrid.formCandidatesCpu)."""
        CrosslinkerSystem.gridFormCount(filCoord, filSegLength, filID, self.gridParams, self.gridDims,
                                        self.gridCellOffsets, self.gridCellContents, self.candCountSeg, formParams)
        CrosslinkerSystem.gridFormScan(self.candCountSeg, self.candBaseSeg, reqFilA, reqFilB, formCounts)
        CrosslinkerSystem.gridFormEmit(filCoord, filSegLength, filID, self.gridParams, self.gridDims,
                                       self.gridCellOffsets, self.gridCellContents, self.candBaseSeg,
                                       self.candCountSeg, reqFilA, reqFilB, formParams)


def _alloc_ck(allocCounts, rankOffsets, freeOffsets, K):
    """(C, K) of an allocator-companion call: allocCounts [0]=C [1]=K when given (host ints),
    else C from freeOffsets (C+1 entries) and K from rankOffsets (reqCap+1 entries)."""
    if allocCounts is not None:
        return int(allocCounts[0]), int(allocCounts[1])
    return freeOffsets.numel() - 1, (rankOffsets.numel() - 1 if K is None else K)


class GrowthSystem:                          # GrowthSystem.java:73-228
    @staticmethod
    def grow(seedNode, monomerCount, coord, uVec, grewFlag, growParams, growCounts):
        _ctx()("sbx_growth_grow", seedNode.numel(), seedNode, monomerCount, coord, uVec, grewFlag, growParams,
               growCounts)

    @staticmethod
    def markSplits(seedNode, monomerCount, coord, uVec, yVec, acceptFlag, reqCoord, reqUVec, reqYVec, splitParams,
                   growCounts):
        _ctx()("sbx_growth_mark_splits", seedNode.numel(), seedNode, monomerCount, coord, uVec, yVec, acceptFlag,
               reqCoord, reqUVec, reqYVec, _n3(reqCoord), splitParams, growCounts)

    @staticmethod
    def splitWire(rankOffsets, freeList, freeOffsets, monomerCount, coord, uVec, end1NbrSlot, end1NbrSide,
                  end2NbrSlot, end2NbrSide, seedNode, splitParams, allocCounts=None, K=None):
        C, K = _alloc_ck(allocCounts, rankOffsets, freeOffsets, K)
        _ctx()("sbx_growth_split_wire", K, C, rankOffsets, freeList, freeOffsets, monomerCount, coord, uVec,
               end1NbrSlot, end1NbrSide, end2NbrSlot, end2NbrSide, seedNode, splitParams)

    @staticmethod
    def recomputeDrag(monomerCount, segLength, end1NbrSlot, end2NbrSlot, bTransGam, bRotGam, bTransDiff, bRotDiff,
                      dragParams, growCounts):
        _ctx()("sbx_growth_recompute_drag", monomerCount.numel(), monomerCount, segLength, end1NbrSlot, end2NbrSlot,
               bTransGam, bRotGam, bTransDiff, bRotDiff, dragParams, growCounts)


class DepolySystem:                          # DepolySystem.java:70-188
    @staticmethod
    def depoly(filState, monomerCount, coord, uVec, end1NbrSlot, returnedMon, deathFlag, depolyParams, depolyCounts):
        _ctx()("sbx_depoly", filState.numel(), filState, monomerCount, coord, uVec, end1NbrSlot, returnedMon,
               deathFlag, depolyParams, depolyCounts)

    @staticmethod
    def depolyProxy(filState, monomerCount, coord, uVec, end1NbrSlot, nucFrac, returnedMon, deathFlag, depolyParams,
                    depolyRateParams, depolyCounts):
        _ctx()("sbx_depoly_proxy", filState.numel(), filState, monomerCount, coord, uVec, end1NbrSlot, nucFrac,
               returnedMon, deathFlag, depolyParams, depolyRateParams, depolyCounts)

    @staticmethod
    def applyDeath(filState, monomerCount, seedNode, end1NbrSlot, end1NbrSide, end2NbrSlot, end2NbrSide,
                   brownTransScale, brownRotScale, deathFlag, depolyCounts=None):
        _ctx()("sbx_depoly_apply_death", filState.numel(), filState, monomerCount, seedNode, end1NbrSlot,
               end1NbrSide, end2NbrSlot, end2NbrSide, brownTransScale, brownRotScale, deathFlag)


class SeveringSystem:                        # SeveringSystem.java:37-98
    @staticmethod
    def cofilinAccumulate(filState, nucFrac, cofFrac, cofilinParams, severCounts):
        _ctx()("sbx_sever_cofilin_accumulate", filState.numel(), filState, nucFrac, cofFrac, cofilinParams,
               severCounts)

    @staticmethod
    def cofilinDissolve(filState, monomerCount, cofFrac, severDeathFlag, severReturnedMon, cofilinParams,
                        severCounts):
        _ctx()("sbx_sever_cofilin_dissolve", filState.numel(), filState, monomerCount, cofFrac, severDeathFlag,
               severReturnedMon, cofilinParams, severCounts)

    @staticmethod
    def nucleateFreshCofilin(rankOffsets, freeList, freeOffsets, cofFrac, allocCounts=None, K=None):
        C, K = _alloc_ck(allocCounts, rankOffsets, freeOffsets, K)
        _ctx()("sbx_sever_nucleate_fresh_cofilin", K, C, rankOffsets, freeList, freeOffsets, cofFrac)


class FilamentBirthSystem:                   # FilamentBirthSystem.java:41-87
    @staticmethod
    def freeFlags(filState, freeCount, allocCounts=None):
        _ctx()("sbx_xlink_free_flags", freeCount.numel(), filState, freeCount)

    @staticmethod
    def freeScatter(filState, freeOffsets, freeList, allocCounts=None):
        _ctx()("sbx_xlink_free_scatter", freeList.numel(), filState, freeOffsets, freeList)

    @staticmethod
    def allocate(reqCoord, reqUVec, reqYVec, rankOffsets, freeList, freeOffsets, coord, uVec, yVec, brownTransScale,
                 brownRotScale, filState, birthParams, allocCounts=None, K=None):
        C, K = _alloc_ck(allocCounts, rankOffsets, freeOffsets, K)
        _ctx()("sbx_birth_allocate", K, C, _n3(reqCoord), reqCoord, reqUVec, reqYVec, rankOffsets, freeList,
               freeOffsets, coord, uVec, yVec, brownTransScale, brownRotScale, filState, birthParams)


class AgingSystem:                           # AgingSystem.java:40-125
    @staticmethod
    def age(filState, nucFrac, agingParams, agingCounts):
        _ctx()("sbx_aging_age", filState.numel(), filState, nucFrac, agingParams, agingCounts)

    @staticmethod
    def growthAtp(grewFlag, monomerCount, nucFrac):
        _ctx()("sbx_aging_growth_atp", grewFlag.numel(), grewFlag, monomerCount, nucFrac)

    @staticmethod
    def splitInheritNuc(rankOffsets, freeList, freeOffsets, nucFrac, allocCounts=None, K=None):
        C, K = _alloc_ck(allocCounts, rankOffsets, freeOffsets, K)
        _ctx()("sbx_aging_split_inherit_nuc", K, C, rankOffsets, freeList, freeOffsets, nucFrac)

    @staticmethod
    def nucleateFreshAtp(rankOffsets, freeList, freeOffsets, nucFrac, allocCounts=None, K=None):
        C, K = _alloc_ck(allocCounts, rankOffsets, freeOffsets, K)
        _ctx()("sbx_aging_nucleate_fresh_atp", K, C, rankOffsets, freeList, freeOffsets, nucFrac)


class FilIDSystem:                           # FilIDSystem.java:30-58
    @staticmethod
    def rounds(n):
        """ceil(log2 n), rounded up to even so the answer lands back in the first buffer."""
        k = 1 if n <= 1 else (n - 1).bit_length()
        return k if k % 2 == 0 else k + 1

    @staticmethod
    def init(filState, end2NbrSlot, ptr, counts=None):
        n = ptr.numel() if counts is None else int(counts[0])
        _ctx()("sbx_filid_init", n, filState, end2NbrSlot, ptr)

    @staticmethod
    def jump(ptrIn, ptrOut, filState, counts=None):
        n = ptrIn.numel() if counts is None else int(counts[0])
        _ctx()("sbx_filid_jump", n, ptrIn, ptrOut, filState)

    @staticmethod
    def compute(filState, end2NbrSlot, ptrA, ptrB):
        """init + rounds(n) jumps ping-ponging A -> B -> A; the result is in ptrA: each active
        segment's chain terminal (its filament id), FREE slots -s-2."""
        n = ptrA.numel()
        FilIDSystem.init(filState, end2NbrSlot, ptrA)
        for r in range(FilIDSystem.rounds(n)):
            src, dst = (ptrA, ptrB) if r % 2 == 0 else (ptrB, ptrA)
            FilIDSystem.jump(src, dst, filState)
        return ptrA


class MotorJointSystem:                      # MotorJointSystem.java:72
    @staticmethod
    def joints(coord, uVec, segLength, bTransGam, bRotGam, forceSum, torqueSum, nucleotideState, jointParams,
               counts=None):
        _ctx()("sbx_motor_joints", _n3(coord), coord, uVec, segLength, bTransGam, bRotGam, forceSum, torqueSum,
               nucleotideState, jointParams)


class DimerCouplingSystem:                   # DimerCouplingSystem.java:83
    @staticmethod
    def couple(coord, uVec, segLength, bTransGam, bRotGam, forceSum, torqueSum, motorA, motorB, parallel,
               dimerParams, boundSeg):
        _ctx()("sbx_dimer_couple", _n3(coord), coord, uVec, segLength, bTransGam, bRotGam, forceSum, torqueSum,
               motorA.numel(), motorA, motorB, parallel, dimerParams, boundSeg)


class MiniFilamentSystem:                    # MiniFilamentSystem.java
    @staticmethod
    def tether(mCoord, mUVec, mSegLength, mBTransGam, mBRotGam, mForceSum, mTorqueSum, bbCoord, bbUVec, bbInvDragY,
               headBackboneSlot, motorA, attachAxial, miniData, miniParams):
        _ctx()("sbx_mini_tether", _n3(mCoord), mCoord, mUVec, mSegLength, mBTransGam, mBRotGam, mForceSum, mTorqueSum,
               _n3(bbCoord), bbCoord, bbUVec, bbInvDragY, headBackboneSlot.numel(), headBackboneSlot, motorA,
               attachAxial, miniData, miniParams)

    @staticmethod
    def backboneGather(bbDimerOffsets, bbDimerList, miniData, bbForceSum, bbTorqueSum, miniCounts=None):
        _ctx()("sbx_mini_backbone_gather", bbDimerOffsets.numel() - 1, bbDimerOffsets, bbDimerList, miniData,
               bbForceSum, bbTorqueSum)


class DeflectionSupport:                     # DeflectionSupport.java:24-58
    @staticmethod
    def seedAccumulators(forceSum, torqueSum, extForce, counts):
        _ctx()("sbx_deflection_seed_accumulators", _n3(forceSum), forceSum, torqueSum, extForce, counts)

    @staticmethod
    def pinEndpoints(coord, uVec, segLength, pinSeg, pinEnd, pinAnchor, counts=None):
        _ctx()("sbx_deflection_pin_endpoints", _n3(coord), coord, uVec, segLength, pinSeg.numel(), pinSeg, pinEnd,
               pinAnchor)


class ThermostatDiag:                        # ThermostatDiag.java:127
    @staticmethod
    def torsionalRestore(uVec, bRotGam, torqueSum, nMotors, coeff, dt):
        _ctx()("sbx_thermostat_torsional_restore", int(nMotors), uVec, bRotGam, torqueSum, float(coeff), float(dt))
