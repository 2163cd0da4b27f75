"""Emit av1b_tables.h: the AV1 specification's normative constant tables.

The tables (cos128, Dr_Intra_Derivative, the smooth weights, the intra edge
kernel, the filter-intra taps, the inter-intra taper, Sgr_Params,
Gaussian_Sequence, Subpel_Filters, Warped_Filters, Upscale_Filter, Div_Lut and
Wedge_Codebook) are part of the bitstream format: a decoder is bit exact only
if every value matches. They are read out of the reference checkout's table
sources (kernels/av1gpu_tables.h, src/core/tables.cpp) so that no value is
retyped, and written here under this library's own names and layout.

    python3 av1ongpu_b200/csrc/gen_tables.py <reference checkout> > av1ongpu_b200/csrc/av1b_tables.h

The output is committed; the build does not run this script.
"""
import re
import sys

if len(sys.argv) != 2:
    raise SystemExit('usage: gen_tables.py <reference checkout>')
REF = sys.argv[1]
tables_h = open(REF + '/kernels/av1gpu_tables.h').read()
tables_cpp = open(REF + '/src/core/tables.cpp').read()
coef_h = open(REF + '/src/frontend/coef_tables.hpp').read()


def numbers(src, decl_regex, count):
    m = re.search(decl_regex + r'[^=]*=\s*\{(.*?)\};', src, re.S)
    if not m:
        raise SystemExit('table not found: ' + decl_regex)
    body = re.sub(r'/\*.*?\*/', '', m.group(1), flags=re.S)
    body = re.sub(r'//[^\n]*', '', body)
    vals = [int(v) for v in re.findall(r'-?\d+', body)]
    if len(vals) != count:
        raise SystemExit('%s: %d values, expected %d' % (decl_regex, len(vals), count))
    return vals


def define(src, name):
    m = re.search(r'#define\s+' + name + r'\s+(-?\d+)', src)
    return int(m.group(1))


def emit(name, ctype, dims, vals, storage='AV1B_TABLE', per_line=16):
    shape = ''.join('[%d]' % d for d in dims)
    out = ['%s %s %s%s = {' % (storage, ctype, name, shape)]
    for i in range(0, len(vals), per_line):
        out.append('    ' + ', '.join(str(v) for v in vals[i:i + per_line]) + ',')
    out.append('};')
    return '\n'.join(out)


parts = []
w = parts.append
w('''/*
 * av1b_tables.h - the AV1 specification's constant tables (generated by
 * gen_tables.py; do not edit). Flattened, one-dimensional where the kernels
 * index them with computed offsets.
 *
 * AV1B_TABLE is the storage class: __device__ for the CUDA build (global
 * memory, read through the L1 so that divergent indices do not serialize the
 * way a __constant__ bank would), plain static const for host code.
 * AV1B_CTABLE: the constant bank, for the small tables a warp reads at one
 * index at a time on the dependency-scheduled path (the mode's angle, its
 * derivative, the edge kernel), whose every L1 miss there is a round trip on
 * the frame's critical path.
 */
#ifndef AV1B_TABLES_H
#define AV1B_TABLES_H
#if defined(__CUDACC__)
#define AV1B_TABLE static __device__ const
#define AV1B_CTABLE static __constant__ const
#else
#define AV1B_TABLE static const
#define AV1B_CTABLE static const
#endif
''')
w('#define AV1B_SINPI_1_9 %d' % define(tables_h, 'AV1G_SINPI_1_9'))
w('#define AV1B_SINPI_2_9 %d' % define(tables_h, 'AV1G_SINPI_2_9'))
w('#define AV1B_SINPI_3_9 %d' % define(tables_h, 'AV1G_SINPI_3_9'))
w('#define AV1B_SINPI_4_9 %d' % define(tables_h, 'AV1G_SINPI_4_9'))
w('')
w('/* cos128(a) = round(4096 cos(a pi / 128)) for a = 0..64 */')
w(emit('kCos128', 'short', [65], numbers(tables_h, r'av1g_tbl_cos128\[65\]', 65)))
w('/* Mode_To_Angle for the thirteen non-CFL intra modes */')
w(emit('kModeAngle', 'short', [13], numbers(tables_h, r'av1g_tbl_mode_to_angle\[13\]', 13), storage='AV1B_CTABLE'))
w('/* Dr_Intra_Derivative, indexed by the angle in degrees (0..89) */')
w(emit('kDrDeriv', 'short', [90], numbers(tables_h, r'av1g_tbl_dr_deriv\[90\]', 90), storage='AV1B_CTABLE'))
sm = []
for n in (4, 8, 16, 32, 64):
    sm += numbers(tables_h, r'av1g_tbl_sm_w%d\[%d\]' % (n, n), n)
w('/* Sm_Weights_Tx_4x4 .. 64x64 back to back: size n starts at n - 4 */')
w(emit('kSmWeights', 'short', [124], sm))
w('/* Intra_Edge_Kernel[strength - 1][tap] */')
w(emit('kEdgeKernel', 'short', [15], numbers(tables_h, r'av1g_tbl_edge_kernel\[3\]\[5\]', 15), storage='AV1B_CTABLE'))
w('/* Intra_Filter_Taps[mode][position 0..7][tap 0..6] */')
w(emit('kFilterIntraTaps', 'signed char', [280],
       numbers(tables_h, r'av1g_tbl_filter_intra\[5\]\[8\]\[7\]', 280), per_line=14))
w('/* Ii_Weights_1d: the inter-intra taper over 128 samples */')
w(emit('kIiWeights', 'unsigned char', [128], numbers(tables_h, r'av1g_tbl_ii_weights\[128\]', 128)))
w('/* Sgr_Params[set]: r0, e0, r1, e1 */')
w(emit('kSgrParams', 'short', [64], numbers(tables_h, r'av1g_tbl_sgr_params\[16\]\[4\]', 64)))
w('/* Gaussian_Sequence */')
w(emit('kGaussianSequence', 'short', [2048],
       numbers(tables_h, r'av1g_tbl_gaussian_sequence\[2048\]', 2048)))
w('/* Subpel_Filters[class][phase][tap]: classes regular, smooth, sharp, bilinear,\n'
  ' * then the 4-tap regular and 4-tap smooth rows (zero padded to 8 taps) */')
w(emit('kSubpelFilters', 'short', [6 * 16 * 8],
       numbers(tables_cpp, r'kSubpelFilters\[kFilterRows\]\[kFilterPhases\]\[kFilterTaps\]',
               6 * 16 * 8), per_line=16))
w('/* Warped_Filters[offset][tap], offset 64 = phase 0 */')
w(emit('kWarpedFilters', 'short', [193 * 8],
       numbers(tables_cpp, r'kWarpedFilters\[kWarpFilterRows\]\[8\]', 193 * 8), per_line=16))
w('/* Upscale_Filter[phase][tap] for superres */')
w(emit('kUpscaleFilter', 'short', [64 * 8],
       numbers(tables_cpp, r'kUpscaleFilter\[64\]\[8\]', 64 * 8), per_line=16))
w('/* Div_Lut: 1/x in Q14 for x in [1, 2) at 8 bits */')
w(emit('kDivLut', 'int', [257], numbers(tables_cpp, r'kDivLut\[257\]', 257)))
m = re.search(r'kWedgeCodebook\[3\]\[16\]\s*=\s*\{(.*?)\};', tables_cpp, re.S)
dirs = {'HORIZONTAL': 0, 'VERTICAL': 1, 'OBLIQUE27': 2, 'OBLIQUE63': 3, 'OBLIQUE117': 4,
        'OBLIQUE153': 5}
codes = [(dirs[d], int(x), int(y)) for d, x, y in
         re.findall(r'\{AV1G_WEDGE_(\w+),\s*(\d+),\s*(\d+)\}', m.group(1))]
if len(codes) != 48:
    raise SystemExit('wedge codebook: %d entries' % len(codes))
w('/* Wedge_Codebook[shape][index]: direction (0 horizontal, 1 vertical, 2..5 oblique\n'
  ' * 27/63/117/153), x offset, y offset in eighths; shapes tall, wide, square */')
w(emit('kWedgeCodebook', 'unsigned char', [48 * 3], [v for c in codes for v in c], per_line=12))


def scan_offsets(fn):
    m = re.search(r'inline int ' + fn + r'\(int lw, int lh\)\s*\{(.*?)\n\}', coef_h, re.S)
    if not m:
        raise SystemExit('scan offsets not found: ' + fn)
    return {int(k, 16): int(v) for k, v in re.findall(r'case (0x[0-9a-f]+): return (-?\d+);', m.group(1))}


n2d, nrow, ncol = 3344, 784, 784
scans = (numbers(coef_h, r'kDefaultScan\[3344\]', n2d) + numbers(coef_h, r'kMrowScan\[784\]', nrow) +
         numbers(coef_h, r'kMcolScan\[784\]', ncol))
w('/* The coefficient scans, positions in raster order of the (at most 32x32)\n'
  ' * coded block: Default_Scan_* (the 2-D classes), then Mrow_Scan_* (vertical\n'
  ' * 1-D types), then Mcol_Scan_* (horizontal 1-D types), each run of sizes back\n'
  ' * to back; kScanOffset gives where a size starts */')
w('#define AV1B_SCAN_ENTRIES %d' % len(scans))
w(emit('kScans', 'unsigned short', [len(scans)], scans))
table = []
for cls, fn, base in ((0, 'default_scan_offset', 0), (1, 'col_scan_offset', n2d + nrow),
                      (2, 'row_scan_offset', n2d)):
    offs = scan_offsets(fn)
    row = [-1] * 16
    for key, v in offs.items():
        lw, lh = key >> 4, key & 15
        row[lw * 4 + lh] = base + v if v >= 0 else -1
    table += row
w('/* kScanOffset[class][lw * 4 + lh]: the start in kScans of the scan of a\n'
  ' * (1 << (lw + 2)) x (1 << (lh + 2)) coded block, lw, lh <= 3; classes 2-D,\n'
  ' * horizontal (column scan), vertical (row scan); -1: no such scan (host table) */')
w(emit('kScanOffset', 'short', [48], table, storage='static const'))
w('#endif /* AV1B_TABLES_H */')
print('\n'.join(parts))
