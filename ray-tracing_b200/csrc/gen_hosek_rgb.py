"""Writes lrt_hosek_rgb.inc: the Hosek-Wilkie RGB sky-model coefficient dataset (Hosek & Wilkie,
"An Analytic Model for Full Spectral Sky-Dome Radiance", 2012; the RGB tables of the model's v1.4a
release, as vendored by the reference in third_party/hosek/ArHosekSkyModelData_RGB.h).

The library cooks the sky state from these numbers exactly as the reference's env_emitter does, so the
tables must hold the same doubles: each value is carried over as the decimal literal it is published as.

    python gen_hosek_rgb.py [path/to/ArHosekSkyModelData_RGB.h]
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT = "/root/reference/third_party/hosek/ArHosekSkyModelData_RGB.h"


def arrays(text):
    out = {}
    for m in re.finditer(r"double\s+(\w+)\[\]\s*=\s*\{(.*?)\};", text, re.S):
        body = re.sub(r"//[^\n]*", "", m.group(2))
        out[m.group(1)] = [v.strip() for v in body.split(",") if v.strip()]
    return out


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else DEFAULT
    with open(src) as f:
        a = arrays(f.read())
    lines = ["// Generated by gen_hosek_rgb.py: Hosek-Wilkie RGB sky-model coefficients (Hosek & Wilkie 2012).",
             "// kHosekRgb[channel]: [albedo 0, 1][turbidity 1..10][6 elevation control points][9 coefficients]",
             "// kHosekRgbRad[channel]: [albedo 0, 1][turbidity 1..10][6 elevation control points]", ""]
    for name, key, n in (("kHosekRgb", "datasetRGB%d", 1080), ("kHosekRgbRad", "datasetRGBRad%d", 120)):
        lines.append("static const double %s[3][%d] = {" % (name, n))
        for c in range(3):
            vals = a[key % (c + 1)]
            assert len(vals) == n, (key % (c + 1), len(vals))
            for v in vals:
                float(v)
            lines.append("    {")
            for i in range(0, n, 6):
                lines.append("        " + ", ".join(vals[i:i + 6]) + ",")
            lines.append("    },")
        lines.append("};")
        lines.append("")
    with open(os.path.join(HERE, "lrt_hosek_rgb.inc"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
