"""Snapshot writer of the reference (main.cu:663-713, compiled in with
GRO_FLAG): one POV-Ray scene text per sample with the big particles of the
slab 1 < z < 3 coloured by colors.cu's neighbour statistics and the small
particles of 1.2 < z < 2.8 in yellow, plus one color_statistics.out line
(time, red, green, blue).  Text output only: no renderer is involved."""
from __future__ import annotations

import numpy as np

COLOR_NAMES = ("Blue", "Green", "Red")

_HEADER = """#include "colors.inc"
global_settings {
\tradiosity{
\t\tpretrace_start 0.08
\t\tpretrace_end   0.01
\t\tcount 150
\t\tnearest_count 10
\t\terror_bound 0.35
\t\trecursion_limit 2
\t\tlow_error_factor 0.5
\t\tgray_threshold 0.0
\t\tminimum_reuse 0.005
\t\tmaximum_reuse 0.2
\t\tbrightness 1
\t\tadc_bailout 0.005
\t}
}
background {White}
camera{
\tangle 90
\tlocation <9,9,15>
\tlook_at <9,9,2>
}
light_source{ <25,25,25> color White}
"""


def write_pov(path: str, rr_big: np.ndarray, rr_sml: np.ndarray, sigma_big: float, sigma_sml: float,
              color_ids: np.ndarray) -> None:
    """snapshot_%d.pov in the reference's format (%8.3f fields)."""
    rr_big = np.asarray(rr_big, np.float32)
    rr_sml = np.asarray(rr_sml, np.float32)
    rb, rs = float(np.float32(sigma_big) * np.float32(0.5)), float(np.float32(sigma_sml) * np.float32(0.5))
    with open(path, "w") as f:
        f.write(_HEADER)
        for (x, y, z), cid in zip(rr_big, color_ids):
            if 1.0 < z < 3.0:
                f.write("sphere{ <%8.3f,%8.3f,%8.3f>, %8.3f pigment {%s} finish { specular 0.5 }}\n"
                        % (x, y, z, rb, COLOR_NAMES[int(cid)]))
        for x, y, z in rr_sml:
            if np.float32(1.2) < z < np.float32(2.8):
                # the reference prints the small particles without commas (main.cu:706-708)
                f.write("sphere{ <%8.3f%8.3f%8.3f>, %8.3f pigment {Yellow} finish { specular 0.5 }}\n" % (x, y, z, rs))


def color_statistics_line(time: float, counts) -> str:
    """One line of color_statistics.out: time, red, green, blue (main.cu:713)."""
    blue, green, red = (int(c) for c in counts)
    return "%f  %d  %d  %d\n" % (time, red, green, blue)
