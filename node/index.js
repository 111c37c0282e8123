// The drop-in `Hush` / `SVGF` classes with the reference's surface (src/index.d.ts:36-83), over the N-API addon
// (hush_node.c) and the CUDA library behind it. GPUTextures become BigInt device addresses of rgba16float images
// (8 bytes per texel, dense rows); the command encoder becomes a CUDA stream handle (BigInt, 0n = default stream).
'use strict';
const native = require('./build/Release/hush_node.node');

// f16 weights as a Uint16Array from an ArrayBuffer, any typed array / DataView, or a base64 string (hush.js:706-717)
function weightsU16(w) {
  if (w === undefined || w === null) return undefined;
  if (typeof w === 'string') {
    const b = Buffer.from(w, 'base64');
    return new Uint16Array(b.buffer.slice(b.byteOffset, b.byteOffset + (b.byteLength & ~1)));
  }
  if (w instanceof Uint16Array) return w;
  if (w instanceof ArrayBuffer) return new Uint16Array(w.slice(0, w.byteLength & ~1));
  if (ArrayBuffer.isView(w)) {
    return new Uint16Array(w.buffer.slice(w.byteOffset, w.byteOffset + (w.byteLength & ~1)));
  }
  throw new Error('Hush: weights must be an ArrayBuffer, a typed array or a base64 string');
}

class Hush {
  // Hush.requiredLimits (hush.js:721, 726): what the device must offer
  static get requiredLimits() { return Object.freeze(native.requiredLimits()); }

  constructor(device, { width, height, exposure = 1, weights, f16 = false } = {}) {
    this.device = device ?? -1;  // a CUDA device ordinal; -1 = the current device
    this._h = native.hushCreate({ width, height, exposure, f16, weights: weightsU16(weights),
                                  device: typeof this.device === 'number' ? this.device : -1 });
    this.width = width;
    this.height = height;
    this._exposure = exposure;
  }

  get exposure() { return this._exposure; }
  set exposure(e) { native.hushSetExposure(this._h, e); this._exposure = e; }

  // denoise(encoder, inputs, timer?) (hush.js:813-822): enqueues the frame on the stream, returns the output address
  denoise(stream, inputs, timer) { return native.hushDenoise(this._h, inputs, stream ?? 0n); }

  // the output of the last denoise(): alternates between two images from frame to frame (hush.js:796-798)
  get output() { return native.hushOutput(this._h); }

  resize(width, height) { native.hushResize(this._h, width, height); this.width = width; this.height = height; }
  reset() { native.hushReset(this._h); }
  destroy() { native.hushDestroy(this._h); }
}

class SVGF {
  constructor(device, width, height, options = {}) {
    this.device = device ?? -1;
    this._s = native.svgfCreate(width, height, options, typeof this.device === 'number' ? this.device : -1);
    this.width = width;
    this.height = height;
  }
  // encode(encoder, inputs + {prevNormalDepth, prevMotion}) (svgf.js:343-378)
  encode(stream, inputs, timer) { return native.svgfEncode(this._s, inputs, stream ?? 0n); }
  get output() { return native.svgfOutput(this._s); }
  resize(width, height) { native.svgfResize(this._s, width, height); this.width = width; this.height = height; }
  reset() { native.svgfReset(this._s); }
  destroy() { native.svgfDestroy(this._s); }
}

// hiddenOf(count) (hush.js:22-25)
function hiddenOf(count) { return native.hiddenOf(count); }

module.exports = { Hush, SVGF, hiddenOf };
