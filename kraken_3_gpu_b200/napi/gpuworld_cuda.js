// gpuworld_cuda.js -- the src/gpu/gpuworld.js surface with CUDA (B200) behind
// it, through the kraken_napi addon.  Drop it next to the reference's
// gpuworld.js (src/gpu/) and point gputrain.js's gpuBackend (and any other
// caller of create / upload / uploadControls / step / download / destroy) at
// this module; the pure functions -- GPU_STRIDES, groupCollPoints,
// packControls, mirrorInto -- are the reference's own, imported unchanged,
// so tools/harness.js's mirror / pack checks keep pinning the same code.
//
// The addon is loaded from $KRAKEN_NAPI, else from build/Release of the
// node-gyp build next to binding.gyp (see INTEGRATION.md).
import { createRequire } from 'node:module';
import { ensureColored } from '../physics/xpbd.js';
import { GPU_STRIDES, groupCollPoints, packControls, mirrorInto } from './gpuworld.js';

export { GPU_STRIDES, groupCollPoints, packControls, mirrorInto };

const require = createRequire(import.meta.url);
const addon = require(process.env.KRAKEN_NAPI || '../../build/Release/kraken_napi.node');
const B = GPU_STRIDES.body, C = GPU_STRIDES.constraint;

export function isAvailable() {
  return addon.deviceCount() > 0;
}

// create(cpu, map): the device world for an XpbdWorld and its map.  The
// WGSL source and WebGPU device arguments of the reference are accepted and
// ignored.
export async function create(cpu, map, _wgslSource, _device) {
  ensureColored(cpu);
  const { order, range } = groupCollPoints(cpu.collPts, cpu.n);
  const coll = new Uint32Array(order.length * 4), collF = new Float32Array(coll.buffer);
  for (let q = 0; q < order.length; q++) {
    const p = cpu.collPts[order[q]];
    coll[4 * q] = p.body; collF[4 * q + 1] = p.lx; collF[4 * q + 2] = p.ly; collF[4 * q + 3] = p.r;
  }
  const rects = new Float32Array(map.rects.length * 4);
  map.rects.forEach((r, i) => rects.set([r.x, r.y, r.w, r.h], 4 * i));
  const nC = cpu.constraints.length;
  const params = { h: cpu.h, substeps: cpu.substeps, iterations: cpu.iterations, linDrag: cpu.linDrag,
                   angDrag: cpu.angDrag, maxSpeed: cpu.maxSpeed, maxAngSpeed: cpu.maxAngSpeed };
  const h = addon.create(params, cpu.n, nC, rects, coll, Uint32Array.from(range));
  return { h, cpu, map, nB: cpu.n, nC, dispatches: 0,
           bodyData: new Float32Array(cpu.n * B), consData: new Float32Array(nC * C),
           forceData: new Float32Array(cpu.n * 4) };
}

// upload(g): the whole CPU world into the 48 B / 80 B / 16 B blocks, then to
// the device (the device re-derives each creature's solve schedule).
export function upload(g) {
  const { cpu, bodyData: bd, consData: cd, forceData: fd } = g;
  const cu = new Uint32Array(cd.buffer);
  for (let i = 0; i < cpu.n; i++) {
    bd.set([cpu.px[i], cpu.py[i], cpu.ppx[i], cpu.ppy[i], cpu.vx[i], cpu.vy[i], cpu.ang[i], cpu.angP[i],
            cpu.av[i], cpu.im[i], cpu.ii[i], 0], i * B);
    fd.set([cpu.fx[i], cpu.fy[i], cpu.tq[i], 0], i * 4);
  }
  cpu.constraints.forEach((c, k) => {
    const o = k * C;
    cu[o] = c.a; cu[o + 1] = c.b >= 0 ? c.b : 0xffffffff; cu[o + 2] = c.type; cu[o + 3] = c.owner;
    cd.set([c.lax, c.lay, c.lbx, c.lby, c.compliance, c.rest, c.target, c.minAngle, c.maxAngle,
            c.lambdaX || 0, c.lambdaY || 0, c.lambda,
            Number.isFinite(c.breakForce) ? Math.min(c.breakForce, 1e30) : 1e30], o + 4);
    cu[o + 17] = c.broken ? 1 : 0; cu[o + 18] = 0; cu[o + 19] = 0;
  });
  const ci = new Uint32Array(33);
  for (let c = 0; c < 16; c++) { ci[c] = cpu.colorOff[c]; ci[16 + c] = cpu.colorCnt[c]; }
  addon.upload(g.h, bd, cd, fd, ci);  // throws Error on a bad body index, as gpuworld.js does
}

export function uploadControls(g) {
  packControls(g.cpu, g.consData);
  addon.uploadControls(g.h, g.consData);
}

export async function step(g) {
  addon.step(g.h, 1);
  g.dispatches += 1;
}

export async function download(g) {
  addon.download(g.h, g.bodyData, g.consData);
  return mirrorInto(g.cpu, g.bodyData, g.consData);
}

export function destroy(g) {
  if (!g) return;
  try { addon.destroy(g.h); } catch (e) { /* already destroyed */ }
}

export async function loadWgsl() {
  return '';  // no shader: the kernels are compiled into libkraken_b200.so
}
