// CudaSolver: the reference's ClothSolver backend (src/backend/solver.ts:5-13)
// running on one B200 through libclosim_cuda.so, loaded as the N-API addon
// built from host/napi (binding.gyp). It is a drop-in for CpuSolver
// (src/backend/cpu-solver.ts:7-49): the same methods, the same error texts,
// and the same aliasing of the caller's scene.
//
// Placement in the reference tree: src/backend/cuda-solver.ts, beside
// cpu-solver.ts; the addon builds to native/build/Release/closim_cuda.node.
//
// Semantics kept from CpuSolver:
// - initialize(scene) keeps the scene by reference (cpu-solver.ts:11-13);
// - step(dt) writes the new state into scene.positions / scene.velocities,
//   which getPositions / getVelocities return (cpu-solver.ts:40-48), so code
//   that reads the scene arrays after a step sees the result;
// - the pin map is read from scene.pinned at every step, because callers
//   mutate it between steps (tests/self-contact.test.ts:73-75);
// - setMaterial stores a copy of the material in the scene (cpu-solver.ts:20-23);
// - pinVertex without a position pins at the current position and enforces
//   all pins on scene.positions (cpu-solver.ts:25-34).
import { createRequire } from "node:module";
import type { ClothSolver } from "./solver.js";
import type { ClothMaterial } from "../physics/types.js";
import type { ClothScene } from "../physics/scene.js";
import { enforcePins } from "../physics/scene.js";
import type { StepStats, StepperOptions } from "../solver/newton.js";
import type { ContactParams } from "../collision/types.js";

/** The addon's exports (host/napi/addon.cc). */
interface CudaAddon {
  create(precision: Precision, device: number): CudaHandle;
  destroy(h: CudaHandle): void;
  initialize(
    h: CudaHandle,
    mesh: {
      count: number;
      triCount: number;
      indices: Uint32Array;
      restPositions: Float32Array;
      invDm: Float32Array;
      areas: Float32Array;
      masses: Float32Array;
    },
    hinges: Int32Array,
    hingeMeta: Float64Array,
    material: ClothMaterial,
    gravity: [number, number, number],
    positions: Float64Array,
    velocities: Float64Array,
  ): void;
  setContact(
    h: CudaHandle,
    params: ContactParams | null,
    floorY: number | null,
    staticPos: Float32Array | null,
    staticIdx: Uint32Array | null,
  ): void;
  setStepperOptions(h: CudaHandle, o: Required<StepperOptions> & { preconditioner: Preconditioner }): void;
  setMaterial(h: CudaHandle, m: ClothMaterial): void;
  setPins(h: CudaHandle, ids: Int32Array, pos: Float64Array): void;
  setState(h: CudaHandle, positions: Float64Array | null, velocities: Float64Array | null): void;
  step(h: CudaHandle, dt: number, positions: Float64Array, velocities: Float64Array): void;
  lastStats(h: CudaHandle): StepStats & { newtonItersUsed: number; armijoTrials: number };
  forward(h: CudaHandle, dt: number, steps: number, checkpointEvery: number, positions: Float64Array): void;
  backward(h: CudaHandle, dLdxN: Float64Array, dLdTheta: Float64Array, dLdv0: Float64Array | null): void;
  membraneHvp(h: CudaHandle, x: Float64Array, p: Float64Array, out: Float64Array): void;
  setNewtonMode(h: CudaHandle, mode: NewtonMode, tol: number): void;
  setGraphMode(h: CudaHandle, on: boolean): void;
  graphInfo(h: CudaHandle): { graphSteps: number; repeats: number };
}

/** Opaque solver handle owned by the addon. */
export type CudaHandle = { readonly __brand: "closim_cuda_handle" };
export type Precision = "fp64" | "mixed";
export type Preconditioner = "jacobi" | "schwarz" | "mas2";
export type NewtonMode = "reference" | "exact";

export interface CudaSolverOptions extends StepperOptions {
  /** "fp64": the reference's arithmetic, op for op; "mixed": FP32 linear solve. */
  precision?: Precision;
  device?: number;
  preconditioner?: Preconditioner;
}

const require = createRequire(import.meta.url);
const cs: CudaAddon = require("../../native/build/Release/closim_cuda.node");

// implicitStep's defaults (src/solver/newton.ts:30-33).
const DEFAULT_STEPPER: Required<StepperOptions> = {
  newtonIters: 10,
  pcgMaxIters: 60,
  gradTol: 1e-5,
  lineSearchIters: 10,
};

function notInitialized(): Error {
  return new Error("CpuSolver not initialized");
}

/** Hinge[] (src/physics/types.ts:29-37) as the flat arrays the C ABI takes. */
function flattenHinges(scene: ClothScene): { ids: Int32Array; meta: Float64Array } {
  const hs = scene.mesh.hinges;
  const ids = new Int32Array(hs.length * 4);
  const meta = new Float64Array(hs.length * 3);
  hs.forEach((h, i) => {
    ids.set([h.v0, h.v1, h.v2, h.v3], i * 4);
    meta.set([h.restAngle, h.edgeLen, h.areaSum], i * 3);
  });
  return { ids, meta };
}

export class CudaSolver implements ClothSolver {
  private scene: ClothScene | null = null;
  private handle: CudaHandle | null;
  lastStats: StepStats | null = null;

  constructor(opts: CudaSolverOptions = {}) {
    this.handle = cs.create(opts.precision ?? "fp64", opts.device ?? 0);
    cs.setStepperOptions(this.handle, {
      newtonIters: opts.newtonIters ?? DEFAULT_STEPPER.newtonIters,
      pcgMaxIters: opts.pcgMaxIters ?? DEFAULT_STEPPER.pcgMaxIters,
      gradTol: opts.gradTol ?? DEFAULT_STEPPER.gradTol,
      lineSearchIters: opts.lineSearchIters ?? DEFAULT_STEPPER.lineSearchIters,
      preconditioner: opts.preconditioner ?? "jacobi",
    });
  }

  private h(): CudaHandle {
    if (!this.handle) throw new Error("CudaSolver was disposed");
    return this.handle;
  }

  initialize(scene: ClothScene): void {
    this.scene = scene;
    const { ids, meta } = flattenHinges(scene);
    cs.initialize(this.h(), scene.mesh, ids, meta, scene.material, scene.gravity, scene.positions, scene.velocities);
    this.sendPins();
    const c = scene.contact;
    cs.setContact(this.h(), c ? c.params : null, c ? c.floorY : null, c ? c.staticPos : null, c ? c.staticIdx : null);
  }

  step(dt: number): void {
    if (!this.scene) throw notInitialized();
    this.sendPins();
    cs.step(this.h(), dt, this.scene.positions, this.scene.velocities);
    this.lastStats = cs.lastStats(this.h());
  }

  setMaterial(material: ClothMaterial): void {
    if (!this.scene) throw notInitialized();
    this.scene.material = { ...material };
    cs.setMaterial(this.h(), this.scene.material);
  }

  pinVertex(vertexId: number, position?: [number, number, number]): void {
    if (!this.scene) throw notInitialized();
    const x = this.scene.positions;
    const p: [number, number, number] = position ?? [x[vertexId * 3], x[vertexId * 3 + 1], x[vertexId * 3 + 2]];
    this.scene.pinned.set(vertexId, p);
    enforcePins(this.scene, x);
    cs.setState(this.h(), x, null);
    this.sendPins();
  }

  unpinVertex(vertexId: number): void {
    this.scene?.pinned.delete(vertexId);
  }

  getPositions(): Float64Array {
    if (!this.scene) throw notInitialized();
    return this.scene.positions;
  }

  getVelocities(): Float64Array {
    if (!this.scene) throw notInitialized();
    return this.scene.velocities;
  }

  /** Uploads scene.positions / scene.velocities after the caller edited them in place. */
  pushState(): void {
    if (!this.scene) throw notInitialized();
    cs.setState(this.h(), this.scene.positions, this.scene.velocities);
  }

  /** Stepper budget and preconditioner (implicitStep's StepperOptions, newton.ts:20-25). */
  setStepperOptions(opts: StepperOptions & { preconditioner?: Preconditioner }): void {
    cs.setStepperOptions(this.h(), {
      newtonIters: opts.newtonIters ?? DEFAULT_STEPPER.newtonIters,
      pcgMaxIters: opts.pcgMaxIters ?? DEFAULT_STEPPER.pcgMaxIters,
      gradTol: opts.gradTol ?? DEFAULT_STEPPER.gradTol,
      lineSearchIters: opts.lineSearchIters ?? DEFAULT_STEPPER.lineSearchIters,
      preconditioner: opts.preconditioner ?? "jacobi",
    });
  }

  /**
   * Newton mode (no counterpart in the reference). "reference", the default,
   * is implicitStep's own linear solve. "exact" solves with the full Hessian to
   * the relative PCG tolerance `tol`, starts Newton from x0 + h v and treats the
   * lagged friction as a frozen potential: with a tight gradTol every step
   * converges, to the same solution in far fewer Newton iterations.
   */
  setNewtonMode(mode: NewtonMode, tol = 1e-6): void {
    cs.setNewtonMode(this.h(), mode, tol);
  }

  /** Graph-captured steps (on by default) or the host-driven step. */
  setGraphMode(on: boolean): void {
    cs.setGraphMode(this.h(), on);
  }

  /** Steps taken as graph replays, and steps repeated host-driven after a buffer grew. */
  graphInfo(): { graphSteps: number; repeats: number } {
    return cs.graphInfo(this.h());
  }

  /** membraneHvp(x, p) (src/physics/fem.ts:108-130) on the GPU. */
  membraneHvp(x: Float64Array, p: Float64Array): Float64Array {
    if (!this.scene) throw notInitialized();
    const out = new Float64Array(x.length);
    cs.membraneHvp(this.h(), x, p, out);
    return out;
  }

  /** Releases the device memory and stream now instead of at garbage collection. */
  dispose(): void {
    if (this.handle) cs.destroy(this.handle);
    this.handle = null;
  }

  // scene.pinned (a Map) as the id / position arrays of cs_set_pins; sent on
  // every step because callers mutate the map between steps.
  private sendPins(): void {
    const pins = this.scene!.pinned;
    const ids = new Int32Array(pins.size);
    const pos = new Float64Array(pins.size * 3);
    let k = 0;
    for (const [id, p] of pins) {
      ids[k] = id;
      pos.set(p, k * 3);
      k++;
    }
    cs.setPins(this.h(), ids, pos);
  }

  /** Handle for the rollout below. */
  get nativeHandle(): CudaHandle {
    return this.h();
  }
}

/** dL/d(C00, C11, G, k_bend) and dL/dv0 of a loss on the final positions. */
export interface RolloutGrad {
  C00: number;
  C11: number;
  G: number;
  kBend: number;
  v0: Float64Array;
}

/**
 * Differentiable rollout with torch.autograd.Function semantics: forward()
 * runs the steps (state checkpointed every `checkpointEvery` steps on the
 * device) and saves what backward() needs; backward(dL/dx_N) returns the
 * gradient with respect to the material parameters and the initial
 * velocities, through the implicit-function theorem on every step (the
 * checkpoint segments are recomputed). The reference has no counterpart.
 */
export class CudaRollout {
  private saved: { n3: number } | null = null;

  constructor(private readonly solver: CudaSolver, private readonly scene: ClothScene) {}

  /** theta = [C00, C11, G, k_bend]; v0: initial velocities (3n). Returns x_N. */
  forward(theta: [number, number, number, number], v0: Float64Array, dt: number, steps: number,
          checkpointEvery = 20): Float64Array {
    const m = this.scene.material;
    this.solver.setMaterial({ ...m, stretchWarp: theta[0], stretchWeft: theta[1], shear: theta[2],
                              bendWarp: theta[3], bendWeft: theta[3] });
    this.scene.velocities.set(v0);
    this.solver.pushState();
    cs.forward(this.solver.nativeHandle, dt, steps, checkpointEvery, this.scene.positions);
    this.saved = { n3: this.scene.positions.length };
    return this.scene.positions;
  }

  backward(dLdxN: Float64Array): RolloutGrad {
    if (!this.saved) throw new Error("backward needs a forward rollout");
    if (dLdxN.length !== this.saved.n3) throw new RangeError("dL/dx_N must hold 3n values");
    const th = new Float64Array(4);
    const dv = new Float64Array(this.saved.n3);
    cs.backward(this.solver.nativeHandle, dLdxN, th, dv);
    return { C00: th[0], C11: th[1], G: th[2], kBend: th[3], v0: dv };
  }
}
