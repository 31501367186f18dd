'use strict';
// CUDA backend of the ashburn-heat-twin live solver for Node: the device half of js/live/solver.js's LiveSolver over
// the N-API binding of libahx.so (ahx_napi.node, built from ahx_napi.cc by node-gyp).
//
// solver.js keeps its domain and parameter code (domain.js, _writeParams, setMet, _setGeometry, _writeColumns, the
// flow-reference logic) and hands the device the byte images it already builds. A LiveSolver constructed with a
// CudaLiveDevice calls, in place of its WebGPU code:
//   _init buffers + pipelines (:137-196)        -> new CudaLiveDevice({ nx, ny, nz, precision, arith, device })
//   _writeParams writeBuffer(P) (:225-242)      -> dev.setParams(this._params)
//   _writeColumns writeBuffer(colv) (:359-376)  -> dev.setColumns(new Uint32Array(buf))
//   _setGeometry ktop + reinit (:323-356)       -> dev.setKtop(Uint32Array.from(ktopS), grew ? Uint32Array.from(old) : null)
//   _reinitFlow (:288-293)                      -> dev.initFlow()
//   resetHeat (:380-386)                        -> dev.clearHeat()
//   resetFlow (:389-398)                        -> dev.initFlow(); dev.clearHeat(); dev.setParity(0)
//   step(n) / _encodeSteps (:401-427)           -> return dev.step(n)          (resolves when the steps have run)
//   read({vol, wind, volMax}) (:439-471)        -> dev.read(this._conv, 255 / vm, this.nzv, vol, wind)
//   benchmark(n) (:474-483)                     -> dev.timeSteps(n)
//   destroy (:485-493)                          -> dev.destroy()
//   _dbg readState / writeState / stepOut / stepAcc / readDbg / clearDbg / stats (:496-578)
//                                               -> dev.readState() / writeState(f, g) / step(n, 'out') /
//                                                  step(n, 'acc') / readDbg() / clearDbg() / stats()
// Each method's C-ABI calls are listed in call_sequences.json.

const path = require('path');

let addon = null;
function binding() {
  if (!addon) {
    // no fallback: without the addon (or without a CUDA device) construction throws
    addon = require(path.join(__dirname, 'build', 'Release', 'ahx_napi.node'));
  }
  return addon;
}

const PRECISIONS = { fp32: 0, fp16: 1, bf16: 2, fp64: 3, fp16g32: 4, bf16g32: 5, fp16sr: 6 };
const ARITH = { exact: 0, fast: 1 };
const MODES = { none: 0, out: 1, acc: 2 };

class CudaLiveDevice {
  /** { nx, ny, nz, precision = 'fp32', arith = 'fast', device = -1 } */
  constructor({ nx, ny, nz, precision = 'fp32', arith = 'fast', device = -1 }) {
    if (!(precision in PRECISIONS)) throw new Error(`live solver: unknown precision ${precision}`);
    if (!(arith in ARITH)) throw new Error(`live solver: unknown arithmetic ${arith}`);
    this.nx = nx; this.ny = ny; this.nz = nz;
    this._h = binding().create(nx, ny, nz, PRECISIONS[precision], device, ARITH[arith]);
    this._destroyed = false;
    const info = binding().info(this._h);
    this.adapterName = `${info.deviceName} (CUDA)`;
  }

  _check() {
    if (this._destroyed) throw new Error('live solver: destroyed');
  }

  // ---- host images
  setParams(bytes) { this._check(); binding().setParams(this._h, bytes); }
  setColumns(colv) { this._check(); binding().setColumns(this._h, colv); }
  setKtop(ktop, oldKtop = null) { this._check(); binding().setKtop(this._h, ktop, oldKtop); }

  // ---- state
  initFlow() { this._check(); binding().initFlow(this._h); }
  clearHeat() { this._check(); binding().clearHeat(this._h); }
  setParity(p) { this._check(); binding().setParity(this._h, p); }

  // ---- stepping: the promise resolves when the GPU has run the n steps (queue.onSubmittedWorkDone)
  step(n, mode = 'none') {
    try { this._check(); } catch (e) { return Promise.reject(e); }
    return binding().step(this._h, Math.max(0, Math.floor(n)), MODES[mode]);
  }

  sync() { this._check(); binding().sync(this._h, -1); }

  // ---- read-back: snapshot of the state the queued steps leave; never blocks stepping
  read(conv, volscale, nzv, vol = true, wind = true) {
    try { this._check(); } catch (e) { return Promise.reject(e); }
    return binding().read(this._h, conv, volscale, nzv, !!vol, !!wind);
  }

  // ---- validation hooks
  readState() { this._check(); return binding().readState(this._h); }
  writeState(f, g) { this._check(); binding().writeState(this._h, f || null, g || null); }
  readDbg() { this._check(); return binding().readDbg(this._h); }
  clearDbg() { this._check(); binding().clearDbg(this._h); }
  stats() { this._check(); return binding().stats(this._h); }
  info() { this._check(); return binding().info(this._h); }
  timeSteps(n) { this._check(); return binding().timeSteps(this._h, n); }
  autotune(stepsPerTrial = 3) { this._check(); return binding().autotune(this._h, stepsPerTrial); }

  destroy() {
    if (this._destroyed) return;
    this._destroyed = true;
    binding().destroy(this._h);
  }
}

module.exports = { CudaLiveDevice, PRECISIONS, ARITH, MODES };
