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


class BrownianForceSystem:                   # BrownianForceSystem.java:183
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


class RigidRodLangevinIntegrationSystem:     # RigidRodLangevinIntegrationSystem.java:279
    @staticmethod
    def integrate(coord, uVec, yVec, forceSum, torqueSum, randForce, randTorque, bTransGam, bRotGam, params,
                  counts=None, coord64=None):
        _ctx()("sbx_integrate", _n3(coord), coord, coord64, uVec, yVec, forceSum, torqueSum, randForce, randTorque,
               bTransGam, bRotGam, params)


class DerivedGeometrySystem:                 # DerivedGeometrySystem.java:386
    @staticmethod
    def derive(coord, uVec, yVec, zVec, end1, end2, segLength, counts=None):
        _ctx()("sbx_derive", _n3(coord), coord, uVec, yVec, zVec, end1, end2, segLength)


class ContainmentSystem:                     # ContainmentSystem.java:390
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


class ThermostatDiag:                        # ThermostatDiag.java:127
    @staticmethod
    def torsionalRestore(uVec, bRotGam, torqueSum, nMotors, coeff, dt):
        _ctx()("sbx_thermostat_torsional_restore", int(nMotors), uVec, bRotGam, torqueSum, float(coeff), float(dt))
