/* Prints sizeof / offsetof of every public struct as JSON; compiled once
 * against the reference's headers (fixture) and once against include/. */
#include <stddef.h>
#include <stdio.h>
#include "wema.h"
#include "iir_filter.h"

#define F(T, m) printf("\"%s.%s\": %zu, ", #T, #m, offsetof(T, m))
#define S(T) printf("\"sizeof(%s)\": %zu, ", #T, sizeof(T))

int main(void) {
    printf("{");
    S(Frame); F(Frame, data); F(Frame, width); F(Frame, height); F(Frame, channels);
    S(Subband); F(Subband, coeffs); F(Subband, width); F(Subband, height);
    S(DWTCoeffs); F(DWTCoeffs, lowpass); F(DWTCoeffs, lowpass_w); F(DWTCoeffs, lowpass_h);
    F(DWTCoeffs, subbands); F(DWTCoeffs, num_levels); F(DWTCoeffs, orig_width); F(DWTCoeffs, orig_height);
    S(TemporalBuffer); F(TemporalBuffer, phase_buffer); F(TemporalBuffer, amplitude);
    F(TemporalBuffer, dc_phase); F(TemporalBuffer, num_positions); F(TemporalBuffer, window_size);
    F(TemporalBuffer, head); F(TemporalBuffer, filled); F(TemporalBuffer, num_levels);
    F(TemporalBuffer, widths); F(TemporalBuffer, heights);
    S(TemporalFilter); F(TemporalFilter, lp_filter); F(TemporalFilter, hp_filter);
    F(TemporalFilter, filter_len); F(TemporalFilter, f_low_norm); F(TemporalFilter, f_high_norm);
    F(TemporalFilter, temporal_levels);
    S(WemaContext); F(WemaContext, width); F(WemaContext, fps); F(WemaContext, amp_factor);
    F(WemaContext, num_levels); F(WemaContext, temporal_window); F(WemaContext, edge_aware);
    F(WemaContext, bilateral_temp); F(WemaContext, color_mode); F(WemaContext, use_iir);
    F(WemaContext, f_low_norm); F(WemaContext, f_high_norm); F(WemaContext, coeffs);
    F(WemaContext, temporal_buf); F(WemaContext, temporal_filt); F(WemaContext, coeffs_cb);
    F(WemaContext, temporal_buf_cr); F(WemaContext, iir_filt); F(WemaContext, iir_filt_cr);
    F(WemaContext, prev_coeffs); F(WemaContext, prev_coeffs_cr); F(WemaContext, gray_in);
    F(WemaContext, delta_phi); F(WemaContext, cb_in); F(WemaContext, delta_cr);
    F(WemaContext, delta_buf); F(WemaContext, guide_buf); F(WemaContext, guided_work);
    S(FFmpegIO); F(FFmpegIO, width); F(FFmpegIO, total_frames); F(FFmpegIO, raw_buffer); F(FFmpegIO, buffer_size);
    S(WemaConfig); F(WemaConfig, amp_factor); F(WemaConfig, temporal_window); F(WemaConfig, ff_codec);
    F(WemaConfig, verbose); F(WemaConfig, use_iir); F(WemaConfig, batch_size); F(WemaConfig, num_threads);
    S(WemaBatchContext); F(WemaBatchContext, batch_size); F(WemaBatchContext, num_positions);
    F(WemaBatchContext, coeffs_batch); F(WemaBatchContext, dwt_batch); F(WemaBatchContext, smooth_buffers);
    F(WemaBatchContext, smooth_buf_stride); F(WemaBatchContext, frames_in_batch); F(WemaBatchContext, warmup_frames);
    S(BiquadCoeffs); S(BiquadState); S(IIRFilterCoeffs); F(IIRFilterCoeffs, sections);
    S(BiquadStateSoA); S(IIRTemporalFilter); F(IIRTemporalFilter, num_positions);
    F(IIRTemporalFilter, state); F(IIRTemporalFilter, state_soa); F(IIRTemporalFilter, warmup_frames);
    F(IIRTemporalFilter, frames_processed); F(IIRTemporalFilter, use_simd);
    printf("\"end\": 0}\n");
    return 0;
}
