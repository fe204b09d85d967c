// The learned moment denoiser of the C ABI (rhgpu_dn_*): its parameters and
// training pairs, forward and backward passes, Adam, and its application to a
// context's moments before the field update.
#include "rhgpu_host.h"

namespace rhh {

const int DN_LOSS_BLOCKS = 296;

// the UMMA B images of every layer (forward and transposed) from the FP32 parameters
int dnRebuildImages(rhgpu_dn* d) {
   for (int l = 0; l < 3; ++l)
      for (int tr = 0; tr < 2; ++tr)
         k_dn_bimage<<<(DN_TAPS * DN_C * DN_C + 255) / 256, 256, 0, d->stream>>>(
             d->params + (size_t)l * DN_LAYER, d->bimg + (size_t)(3 * tr + l) * (TC_BIMG / 2), tr);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

// one convolution layer on the tensor cores (k_dn_conv_tc): layer l, forward or
// transposed (the data gradient); `err` receives RHGPU_DEVERR_DENOISER
int dnConv(rhgpu_dn* d, cudaStream_t st, bool transposed, int l, const unsigned* in, const float* bias, int mode,
           unsigned* out, const unsigned* mask, float* out32, const float* res, const DnMoments& mom, unsigned* err) {
   static bool raised[64][2] = {};
   if (d->device < 0 || d->device >= 64) return fail(RHGPU_ERR_CUDA, "denoiser: device index out of range");
   if (!raised[d->device][transposed]) {
      RH_CUDA(cudaFuncSetAttribute(transposed ? k_dn_conv_tc<true> : k_dn_conv_tc<false>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TC_SMEM));
      raised[d->device][transposed] = true;
   }
   const dim3 grid((unsigned)((d->g.nx + TC_BX - 1) / TC_BX), (unsigned)((d->g.ny + TC_BY - 1) / TC_BY),
                   (unsigned)((d->g.nz + TC_ZC - 1) / TC_ZC));
   const __nv_bfloat16* img = d->bimg + (size_t)((transposed ? 3 : 0) + l) * (TC_BIMG / 2);
   if (transposed)
      k_dn_conv_tc<true><<<grid, TC_THREADS, TC_SMEM, st>>>(d->g, in, img, bias, mode, out, mask, out32, res, mom, err);
   else
      k_dn_conv_tc<false><<<grid, TC_THREADS, TC_SMEM, st>>>(d->g, in, img, bias, mode, out, mask, out32, res, mom, err);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

// the convolutions' device error word, read and cleared (after a synchronisation of d->stream)
int dnCheckError(rhgpu_dn* d) {
   unsigned w = 0;
   RH_CUDA(cudaMemcpyAsync(&w, d->err, sizeof w, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   if (w) {
      RH_CUDA(cudaMemsetAsync(d->err, 0, sizeof w, d->stream));
      return fail(RHGPU_ERR_DEVICE, "denoiser: a convolution's wait on its tensor-core work ran out");
   }
   return RHGPU_OK;
}

// forward of the network on d->res (normalized FP32 input) into d->out32
int dnForward(rhgpu_dn* d) {
   const long long N = d->g.N;
   k_dn_res_to_act<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, d->res, d->act[0]);
   const float* b0 = d->params + DN_TAPS * DN_C * DN_C;
   const float* b1 = d->params + DN_LAYER + DN_TAPS * DN_C * DN_C;
   const float* b2 = d->params + 2 * DN_LAYER + DN_TAPS * DN_C * DN_C;
   int rc = dnConv(d, d->stream, false, 0, d->act[0], b0, 0, d->act[1], nullptr, nullptr, nullptr, DnMoments{}, d->err);
   if (!rc) rc = dnConv(d, d->stream, false, 1, d->act[1], b1, 0, d->act[2], nullptr, nullptr, nullptr, DnMoments{}, d->err);
   if (!rc) rc = dnConv(d, d->stream, false, 2, d->act[2], b2, 3, nullptr, nullptr, d->out32, d->res, DnMoments{}, d->err);
   return rc;
}

// loss against target (normalized FP32, N x 4) and the gradient of all parameters into d->grad
int dnBackward(rhgpu_dn* d, const float* target, double* loss) {
   const long long N = d->g.N;
   // voxels in the loss: all but the masked border of the non-periodic faces
   long long in = 1;
   const int nn[3] = {d->g.nx, d->g.ny, d->g.nz};
   for (int a = 0; a < 3; ++a) in *= d->g.per[a] ? nn[a] : std::max(0, nn[a] - 2 * d->border);
   if (in < 1) return fail(RHGPU_ERR_STATE, "dn_train: the loss border leaves no voxel");
   k_dn_loss<<<DN_LOSS_BLOCKS, 256, 0, d->stream>>>(d->g, d->out32, target, 1.0 / (4.0 * (double)in), d->dY[2], d->lossPart,
                                                   d->border);
   const unsigned wb = (unsigned)((N + DN_WGRAD_VOX - 1) / DN_WGRAD_VOX);
   for (int l = 2; l >= 0; --l) {
      k_dn_wgrad<<<dim3(wb, DN_TAPS), 32 * DN_WARPS, 0, d->stream>>>(d->g, d->act[l], d->dY[l], d->part);
      k_dn_reduce_rows<<<(DN_TAPS * DN_C * DN_C + 255) / 256, 256, 0, d->stream>>>(d->part, wb, DN_TAPS * DN_C * DN_C,
                                                                                  d->grad + (size_t)l * DN_LAYER);
      k_dn_bgrad<<<wb, 256, 0, d->stream>>>(d->g, d->dY[l], d->part);
      k_dn_reduce_rows<<<1, DN_C, 0, d->stream>>>(d->part, wb, DN_C, d->grad + (size_t)l * DN_LAYER + DN_TAPS * DN_C * DN_C);
      if (l > 0)
         if (int rc = dnConv(d, d->stream, true, l, d->dY[l], nullptr, 2, d->dY[l - 1], d->act[l], nullptr, nullptr,
                             DnMoments{}, d->err))
            return rc;
   }
   RH_CUDA(cudaGetLastError());
   std::vector<double> lp(DN_LOSS_BLOCKS);
   RH_CUDA(cudaMemcpyAsync(lp.data(), d->lossPart, sizeof(double) * DN_LOSS_BLOCKS, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   double a = 0.0;
   for (double x : lp) a += x;
   if (loss) *loss = a / (4.0 * (double)in);
   return RHGPU_OK;
}

// host moments in the ABI layout (rho N, Ji interleaved 3N) -> device planar scratch (acc)
int dnUploadMoments(rhgpu_dn* d, const double* rho, const double* ji, double* planar) {
   const long long N = d->g.N;
   std::vector<double> h(4 * (size_t)N);
   for (long long n = 0; n < N; ++n) {
      h[n] = rho[n];
      for (int l = 0; l < 3; ++l) h[(1 + l) * N + n] = ji[3 * n + l];
   }
   RH_CUDA(cudaMemcpyAsync(planar, h.data(), sizeof(double) * 4 * N, cudaMemcpyHostToDevice, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

// the network on planar device moments (rho N, J 3 x N), in place: the first layer
// reads and normalizes them, the last adds its output to their normalized values
// and scales back (rho clamped at minRho), in three launches
int dnApplyMoments(rhgpu_dn* d, cudaStream_t st, double* rho, double* J, double minRho, unsigned* err) {
   const long long N = d->g.N;
   const DnMoments mom{rho, J, d->sr, d->sj, 1.0 / d->sr, 1.0 / d->sj, minRho, N, d->vel, d->keep};
   const float* b0 = d->params + DN_TAPS * DN_C * DN_C;
   const float* b1 = d->params + DN_LAYER + DN_TAPS * DN_C * DN_C;
   const float* b2 = d->params + 2 * DN_LAYER + DN_TAPS * DN_C * DN_C;
   int rc = dnConv(d, st, false, 0, nullptr, b0, 0, d->act[1], nullptr, nullptr, nullptr, mom, err);
   if (!rc) rc = dnConv(d, st, false, 1, d->act[1], b1, 0, d->act[2], nullptr, nullptr, nullptr, DnMoments{}, err);
   if (!rc) rc = dnConv(d, st, false, 2, d->act[2], b2, 4, nullptr, nullptr, nullptr, nullptr, mom, err);
   return rc;
}

// the denoiser on the context's moments (device, on the context's stream), before the field update
int dnApplyCtx(rhgpu_ctx* c) {
   RH_TIME(c, "dn_apply");
   return dnApplyMoments(c->dn, c->stream, c->f.cellRho, c->f.cellJi, c->P.min_ion_charge_density, c->err);
}

}  // namespace rhh

extern "C" {

int rhgpu_dn_create(int32_t nx, int32_t ny, int32_t nz, const int32_t* periodic, int32_t pair_capacity, int32_t device,
                    rhgpu_dn** out) {
   if (!out || !periodic || nx < 1 || ny < 1 || nz < 1 || pair_capacity < 0) return fail(RHGPU_ERR_ARG, "dn_create: bad arguments");
   RH_CUDA(cudaSetDevice(device));
   rhgpu_dn* d = new rhgpu_dn();
   d->device = device;
   d->g.nx = nx; d->g.ny = ny; d->g.nz = nz;
   for (int a = 0; a < 3; ++a) d->g.per[a] = periodic[a] ? 1 : 0;
   d->g.N = (long long)nx * ny * nz;
   const long long N = d->g.N;
   d->pairCap = pair_capacity;
   d->partRows = (N + DN_WGRAD_VOX - 1) / DN_WGRAD_VOX;
   int rc = RHGPU_OK;
   auto alloc = [&](void** p, size_t bytes) {
      if (rc) return;
      if (cudaMalloc(p, bytes) != cudaSuccess) rc = fail(RHGPU_ERR_NOMEM, "dn_create: cudaMalloc");
      else cudaMemset(*p, 0, bytes);
   };
   if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "dn_create: stream");
   alloc((void**)&d->params, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->grad, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->m, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->v, sizeof(float) * DN_PARAMS);
   alloc((void**)&d->mask, DN_PARAMS);
   alloc((void**)&d->bimg, 6 * (size_t)TC_BIMG);
   alloc((void**)&d->err, sizeof(unsigned));
   for (int l = 0; l < 3; ++l) {
      alloc((void**)&d->act[l], sizeof(unsigned) * 8 * N);
      alloc((void**)&d->dY[l], sizeof(unsigned) * 8 * N);
   }
   alloc((void**)&d->res, sizeof(float) * 4 * N);
   alloc((void**)&d->out32, sizeof(float) * 4 * N);
   alloc((void**)&d->part, sizeof(float) * d->partRows * DN_TAPS * DN_C * DN_C);
   alloc((void**)&d->lossPart, sizeof(double) * DN_LOSS_BLOCKS);
   alloc((void**)&d->acc, sizeof(double) * std::max(4 * N, 4LL * 64));   // also k_dn_err's 64 x 4 partials
   if (pair_capacity > 0) {
      alloc((void**)&d->pairIn, sizeof(float) * 4 * N * pair_capacity);
      alloc((void**)&d->pairOut, sizeof(float) * 4 * N * pair_capacity);
   }
   if (!rc) {
      // trainable entries: layer 0 reads 4 channels, layer 2 writes 4 channels
      std::vector<unsigned char> mk(DN_PARAMS, 0);
      for (int l = 0; l < 3; ++l)
         for (int t = 0; t < DN_TAPS; ++t)
            for (int ci = 0; ci < DN_C; ++ci)
               for (int co = 0; co < DN_C; ++co)
                  mk[(size_t)l * DN_LAYER + (t * DN_C + ci) * DN_C + co] = (l == 0 ? ci < 4 : true) && (l == 2 ? co < 4 : true);
      for (int l = 0; l < 3; ++l)
         for (int co = 0; co < DN_C; ++co) mk[(size_t)l * DN_LAYER + DN_TAPS * DN_C * DN_C + co] = l == 2 ? co < 4 : 1;
      if (cudaMemcpy(d->mask, mk.data(), DN_PARAMS, cudaMemcpyHostToDevice) != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "dn_create: mask");
   }
   if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = fail(RHGPU_ERR_CUDA, "dn_create: sync");
   if (rc) {
      rhgpu_dn_destroy(d);
      return rc;
   }
   *out = d;
   return RHGPU_OK;
}

int rhgpu_dn_destroy(rhgpu_dn* d) {
   if (!d) return RHGPU_OK;
   cudaSetDevice(d->device);
   if (d->stream) cudaStreamSynchronize(d->stream);
   cudaFree(d->params); cudaFree(d->grad); cudaFree(d->m); cudaFree(d->v); cudaFree(d->mask); cudaFree(d->bimg); cudaFree(d->err);
   for (int l = 0; l < 3; ++l) { cudaFree(d->act[l]); cudaFree(d->dY[l]); }
   cudaFree(d->res); cudaFree(d->out32); cudaFree(d->part); cudaFree(d->lossPart); cudaFree(d->acc);
   cudaFree(d->pairIn); cudaFree(d->pairOut);
   cudaFree(d->fullAcc); cudaFree(d->fullIn); cudaFree(d->fullOut); cudaFree(d->keep);
   if (d->stream) cudaStreamDestroy(d->stream);
   delete d;
   return RHGPU_OK;
}

int rhgpu_dn_set_params(rhgpu_dn* d, const float* p, int64_t n) {
   if (!d || !p || n != DN_PARAMS) return fail(RHGPU_ERR_ARG, "dn_set_params: needs RHGPU_DN_PARAMS floats");
   RH_CUDA(cudaSetDevice(d->device));
   std::vector<unsigned char> mk(DN_PARAMS);
   RH_CUDA(cudaMemcpy(mk.data(), d->mask, DN_PARAMS, cudaMemcpyDeviceToHost));
   std::vector<float> h(p, p + n);
   for (int64_t e = 0; e < n; ++e) if (!mk[e]) h[e] = 0.f;
   RH_CUDA(cudaMemcpyAsync(d->params, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, d->stream));
   RH_CUDA(cudaMemsetAsync(d->m, 0, sizeof(float) * n, d->stream));
   RH_CUDA(cudaMemsetAsync(d->v, 0, sizeof(float) * n, d->stream));
   d->adamStep = 0;
   int rc = dnRebuildImages(d);
   if (rc) return rc;
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_get_params(rhgpu_dn* d, float* p, int64_t n) {
   if (!d || !p || n != DN_PARAMS) return fail(RHGPU_ERR_ARG, "dn_get_params: needs RHGPU_DN_PARAMS floats");
   RH_CUDA(cudaSetDevice(d->device));
   RH_CUDA(cudaMemcpyAsync(p, d->params, sizeof(float) * n, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_set_scales(rhgpu_dn* d, double rho_scale, double j_scale) {
   if (!d || !(rho_scale > 0) || !(j_scale > 0)) return fail(RHGPU_ERR_ARG, "dn_set_scales: scales must be positive");
   d->sr = rho_scale;
   d->sj = j_scale;
   return RHGPU_OK;
}

int rhgpu_dn_set_velocity_form(rhgpu_dn* d, int32_t enabled) {
   if (!d) return fail(RHGPU_ERR_ARG, "dn_set_velocity_form: null denoiser");
   d->vel = enabled ? 1 : 0;
   return RHGPU_OK;
}

int rhgpu_dn_set_keep_mask(rhgpu_dn* d, const uint8_t* keep) {
   if (!d) return fail(RHGPU_ERR_ARG, "dn_set_keep_mask: null denoiser");
   RH_CUDA(cudaSetDevice(d->device));
   if (!keep) {
      RH_CUDA(cudaStreamSynchronize(d->stream));
      cudaFree(d->keep);
      d->keep = nullptr;
      return RHGPU_OK;
   }
   if (!d->keep) RH_CUDA(cudaMalloc(&d->keep, (size_t)d->g.N));
   RH_CUDA(cudaMemcpyAsync(d->keep, keep, (size_t)d->g.N, cudaMemcpyHostToDevice, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_apply(rhgpu_dn* d, const double* rho_in, const double* ji_in, double* rho_out, double* ji_out, double min_rho) {
   if (!d || !rho_in || !ji_in || !rho_out || !ji_out) return fail(RHGPU_ERR_ARG, "dn_apply: bad arguments");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   int rc = dnUploadMoments(d, rho_in, ji_in, d->acc);
   if (rc) return rc;
   rc = dnApplyMoments(d, d->stream, d->acc, d->acc + N, min_rho, d->err);
   if (!rc) rc = dnCheckError(d);
   if (rc) return rc;
   std::vector<double> h(4 * (size_t)N);
   RH_CUDA(cudaMemcpyAsync(h.data(), d->acc, sizeof(double) * 4 * N, cudaMemcpyDeviceToHost, d->stream));
   RH_CUDA(cudaStreamSynchronize(d->stream));
   for (long long v = 0; v < N; ++v) {
      rho_out[v] = h[v];
      for (int l = 0; l < 3; ++l) ji_out[3 * v + l] = h[(1 + l) * N + v];
   }
   return RHGPU_OK;
}

int rhgpu_dn_loss_grad(rhgpu_dn* d, const double* rho_in, const double* ji_in, const double* rho_t, const double* ji_t,
                       double* loss, float* grad) {
   if (!d || !rho_in || !ji_in || !rho_t || !ji_t) return fail(RHGPU_ERR_ARG, "dn_loss_grad: bad arguments");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   int rc = dnUploadMoments(d, rho_t, ji_t, d->acc);
   if (rc) return rc;
   k_dn_norm<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, d->acc, d->acc + N, 1.0 / d->sr, 1.0 / d->sj, d->vel, d->out32);
   // target kept in dY[0]'s storage as FP32 (N x 4 floats fit in 8 u32 per voxel)
   float* target = reinterpret_cast<float*>(d->dY[0]);
   RH_CUDA(cudaMemcpyAsync(target, d->out32, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
   rc = dnUploadMoments(d, rho_in, ji_in, d->acc);
   if (rc) return rc;
   k_dn_norm<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, d->acc, d->acc + N, 1.0 / d->sr, 1.0 / d->sj, d->vel, d->res);
   rc = dnForward(d);
   if (rc) return rc;
   // the loss kernel reads the target before the backward overwrites dY[0]
   float* tcopy = reinterpret_cast<float*>(d->acc);
   RH_CUDA(cudaMemcpyAsync(tcopy, target, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
   rc = dnBackward(d, tcopy, loss);
   if (!rc) rc = dnCheckError(d);
   if (rc) return rc;
   if (grad) {
      RH_CUDA(cudaMemcpyAsync(grad, d->grad, sizeof(float) * DN_PARAMS, cudaMemcpyDeviceToHost, d->stream));
      RH_CUDA(cudaStreamSynchronize(d->stream));
   }
   return RHGPU_OK;
}

// the normalized moments of a fast-path context (4 x N floats, voxel-major):
// one in `factor` of its particles (from `offset`) with weights times factor,
// or all (factor 1); acc is 4 x N doubles of scratch
int dnDepositSample(rhgpu_dn* d, rhgpu_ctx* c, int factor, int offset, double* acc, float* out) {
   const long long N = c->g.N;
   RH_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * 4 * N, d->stream));
   for (int s = 0; s < c->ns; ++s) {
      if (!c->sp[s].accumulate) continue;
      const SegHost& h = c->seg[s];
      if (!h.a[h.cur][0]) continue;
      k_dn_subsample_deposit<<<(unsigned)c->fg.NS, 128, 0, d->stream>>>(c->g, c->fg, segView(h, h.cur), h.base,
                                                                       c->sp[s].q, factor, offset, acc);
   }
   k_dn_subsample_finish<<<blocks1d(N, 256), 256, 0, d->stream>>>(N, acc, c->g.dV, c->P.min_ion_charge_density,
                                                                 1.0 / d->sr, 1.0 / d->sj, d->vel, out);
   RH_CUDA(cudaGetLastError());
   return RHGPU_OK;
}

int rhgpu_dn_add_crops(rhgpu_dn* d, rhgpu_ctx* c, int32_t factor, int32_t offset, int32_t ncrops, const int32_t* origins) {
   if (!d || !c || factor < 1 || offset < 0 || offset >= factor || ncrops < 1 || !origins)
      return fail(RHGPU_ERR_ARG, "dn_add_crops: bad arguments");
   if (d->pairCap < 1) return fail(RHGPU_ERR_STATE, "dn_add_crops: created without pair capacity");
   if (c->path != RHGPU_PATH_FAST) return fail(RHGPU_ERR_STATE, "dn_add_crops: the context must use RHGPU_PATH_FAST");
   if (c->device != d->device) return fail(RHGPU_ERR_ARG, "dn_add_crops: the device differs");
   for (int q = 0; q < ncrops; ++q) {
      const int* o = origins + 3 * q;
      if (o[0] < 0 || o[1] < 0 || o[2] < 0 || o[0] + d->g.nx > c->g.nx || o[1] + d->g.ny > c->g.ny ||
          o[2] + d->g.nz > c->g.nz)
         return fail(RHGPU_ERR_ARG, "dn_add_crops: a crop leaves the context's grid");
   }
   RH_CUDA(cudaSetDevice(d->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   const long long NF = c->g.N;
   if (d->fullN != NF) {
      cudaFree(d->fullAcc); cudaFree(d->fullIn); cudaFree(d->fullOut);
      d->fullAcc = nullptr; d->fullIn = nullptr; d->fullOut = nullptr;
      d->fullN = 0;
      RH_CUDA(cudaMalloc(&d->fullAcc, sizeof(double) * 4 * NF));
      RH_CUDA(cudaMalloc(&d->fullIn, sizeof(float) * 4 * NF));
      RH_CUDA(cudaMalloc(&d->fullOut, sizeof(float) * 4 * NF));
      d->fullN = NF;
   }
   int rc = dnDepositSample(d, c, factor, offset, d->fullAcc, d->fullIn);
   if (!rc) rc = dnDepositSample(d, c, 1, 0, d->fullAcc, d->fullOut);
   if (rc) return rc;
   const long long N = d->g.N;
   for (int q = 0; q < ncrops; ++q) {
      const int* o = origins + 3 * q;
      float* in = d->pairIn + (size_t)d->pairNext * 4 * N;
      float* tg = d->pairOut + (size_t)d->pairNext * 4 * N;
      k_dn_crop<<<blocks1d(N, 256), 256, 0, d->stream>>>(d->fullIn, c->g.nx, c->g.ny, d->g, o[0], o[1], o[2], in);
      k_dn_crop<<<blocks1d(N, 256), 256, 0, d->stream>>>(d->fullOut, c->g.nx, c->g.ny, d->g, o[0], o[1], o[2], tg);
      d->pairNext = (d->pairNext + 1) % d->pairCap;
      d->pairCount = std::min(d->pairCount + 1, d->pairCap);
   }
   RH_CUDA(cudaGetLastError());
   RH_CUDA(cudaStreamSynchronize(d->stream));
   return RHGPU_OK;
}

int rhgpu_dn_set_loss_border(rhgpu_dn* d, int32_t border) {
   if (!d || border < 0) return fail(RHGPU_ERR_ARG, "dn_set_loss_border: bad arguments");
   d->border = border;
   return RHGPU_OK;
}

int rhgpu_dn_add_pair(rhgpu_dn* d, rhgpu_ctx* c, int32_t factor, int32_t offset) {
   if (!d || !c || factor < 1 || offset < 0 || offset >= factor) return fail(RHGPU_ERR_ARG, "dn_add_pair: bad arguments");
   if (d->pairCap < 1) return fail(RHGPU_ERR_STATE, "dn_add_pair: created without pair capacity");
   if (c->path != RHGPU_PATH_FAST) return fail(RHGPU_ERR_STATE, "dn_add_pair: the context must use RHGPU_PATH_FAST");
   if (c->g.nx != d->g.nx || c->g.ny != d->g.ny || c->g.nz != d->g.nz || c->device != d->device)
      return fail(RHGPU_ERR_ARG, "dn_add_pair: grid or device differs");
   RH_CUDA(cudaSetDevice(d->device));
   RH_CUDA(cudaStreamSynchronize(c->stream));
   const long long N = d->g.N;
   float* in = d->pairIn + (size_t)d->pairNext * 4 * N;
   float* tg = d->pairOut + (size_t)d->pairNext * 4 * N;
   // input: one in `factor` particles, weights times factor; target: all particles,
   // by the same deposit of the same state
   int rc = dnDepositSample(d, c, factor, offset, d->acc, in);
   if (!rc) rc = dnDepositSample(d, c, 1, 0, d->acc, tg);
   if (rc) return rc;
   RH_CUDA(cudaStreamSynchronize(d->stream));
   d->pairNext = (d->pairNext + 1) % d->pairCap;
   d->pairCount = std::min(d->pairCount + 1, d->pairCap);
   return RHGPU_OK;
}

int rhgpu_dn_train(rhgpu_dn* d, int32_t iterations, float lr, double* mean_loss) {
   if (!d || iterations < 0 || !(lr > 0)) return fail(RHGPU_ERR_ARG, "dn_train: bad arguments");
   if (d->pairCount < 1) return fail(RHGPU_ERR_STATE, "dn_train: no training pairs");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   double tot = 0.0;
   const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
   for (int it = 0; it < iterations; ++it) {
      d->rng = d->rng * 6364136223846793005ull + 1442695040888963407ull;
      const int p = (int)((d->rng >> 33) % (unsigned long long)d->pairCount);
      RH_CUDA(cudaMemcpyAsync(d->res, d->pairIn + (size_t)p * 4 * N, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
      int rc = dnForward(d);
      if (rc) return rc;
      double l = 0.0;
      rc = dnBackward(d, d->pairOut + (size_t)p * 4 * N, &l);
      if (rc) return rc;
      tot += l;
      d->adamStep += 1;
      const float c1 = 1.f - std::pow(b1, (float)d->adamStep), c2 = 1.f - std::pow(b2, (float)d->adamStep);
      k_dn_adam<<<(DN_PARAMS + 255) / 256, 256, 0, d->stream>>>(d->params, d->grad, d->m, d->v, d->mask, DN_PARAMS, lr, b1, b2,
                                                               eps, c1, c2);
      rc = dnRebuildImages(d);
      if (rc) return rc;
   }
   RH_CUDA(cudaStreamSynchronize(d->stream));
   if (int rc = dnCheckError(d)) return rc;
   if (mean_loss) *mean_loss = iterations ? tot / iterations : 0.0;
   return RHGPU_OK;
}

int rhgpu_set_denoiser(rhgpu_ctx* c, rhgpu_dn* d, int32_t enabled) {
   if (!c) return fail(RHGPU_ERR_ARG, "set_denoiser: null context");
   if (d && (c->g.nx != d->g.nx || c->g.ny != d->g.ny || c->g.nz != d->g.nz || c->device != d->device ||
             c->g.per[0] != d->g.per[0] || c->g.per[1] != d->g.per[1] || c->g.per[2] != d->g.per[2]))
      return fail(RHGPU_ERR_ARG, "set_denoiser: grid or device differs");
   c->dn = d;
   c->dnOn = d && enabled;
   return RHGPU_OK;
}

int rhgpu_dn_pair_error(rhgpu_dn* d, int32_t pair, double* out4) {
   if (!d || !out4 || pair < 0 || pair >= d->pairCount) return fail(RHGPU_ERR_ARG, "dn_pair_error: bad arguments");
   RH_CUDA(cudaSetDevice(d->device));
   const long long N = d->g.N;
   const float* in = d->pairIn + (size_t)pair * 4 * N;
   const float* tg = d->pairOut + (size_t)pair * 4 * N;
   RH_CUDA(cudaMemcpyAsync(d->res, in, sizeof(float) * 4 * N, cudaMemcpyDeviceToDevice, d->stream));
   int rc = dnForward(d);
   if (rc) return rc;
   std::vector<double> h(4 * 64);
   double r[2][4];
   for (int which = 0; which < 2; ++which) {
      k_dn_err<<<64, 256, 0, d->stream>>>(N, which ? d->out32 : in, tg, d->acc);
      RH_CUDA(cudaGetLastError());
      RH_CUDA(cudaMemcpyAsync(h.data(), d->acc, sizeof(double) * 4 * 64, cudaMemcpyDeviceToHost, d->stream));
      RH_CUDA(cudaStreamSynchronize(d->stream));
      for (int q = 0; q < 4; ++q) {
         r[which][q] = 0.0;
         for (int b = 0; b < 64; ++b) r[which][q] += h[b * 4 + q];
      }
   }
   out4[0] = std::sqrt(r[0][0] / r[0][1]);   // raw rho
   out4[1] = std::sqrt(r[0][2] / r[0][3]);   // raw J
   out4[2] = std::sqrt(r[1][0] / r[1][1]);   // denoised rho
   out4[3] = std::sqrt(r[1][2] / r[1][3]);   // denoised J
   return RHGPU_OK;
}

int rhgpu_dn_num_pairs(rhgpu_dn* d, int32_t* n_out, int32_t* newest) {
   if (!d || !n_out || !newest) return fail(RHGPU_ERR_ARG, "dn_num_pairs: bad arguments");
   *n_out = d->pairCount;
   *newest = d->pairCount ? (d->pairNext + d->pairCap - 1) % d->pairCap : -1;
   return RHGPU_OK;
}

}  // extern "C"
