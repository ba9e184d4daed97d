"""Generate the display golden values of the reference workspace from its own headers.

Reads, as text, the reference's palette table and display defaults and writes
display_reference.json:

  palettes        the 14 five-stop wave palettes of Main_header/WavePalettes.h:11-26
  state_defaults  the in-class defaults of the display members of Seis3D_State
                  (include/Seis3D_Sim.h:110-160) and VolumeCamera3D (:25-28)
  limits          maxVolumeAxis3D / maxVolumeOutput3D (include/Common3D.h:11-12)

    python tests/golden/make_display_golden.py [REFERENCE_ROOT]   (default /root/reference)
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# Display members of Seis3D_State that the renderer turns into uniforms.
STATE_FIELDS = ["displayMode3D", "waveStyle3D", "modelStyle3D", "component3D", "materialRangeAuto3D",
                "materialRange3D", "manualMaterialRange3D", "waveOpacity3D", "waveThreshold3D", "modelOpacity3D",
                "waveGamma3D", "materialBrightness3D", "gain3D", "showBoundary3D", "boundaryOpacity3D",
                "volumeOpacity3D", "volumeThreshold3D", "volumeSampling3D", "volumeSharpness3D", "volumeGain3D",
                "volumeSizeCompensation3D", "volumeRequestedWidth3D", "volumeRequestedHeight3D"]
CAMERA_FIELDS = ["yaw3D", "pitch3D", "distance3D"]


def number(token: str) -> float:
    token = token.strip()
    if token in ("true", "false"):
        return 1.0 if token == "true" else 0.0
    return float(token.rstrip("fF"))


def initialisers(text: str) -> dict:
    """name -> value(s) of every `name = v` / `name[n] = {a, b}` declarator in `text`."""
    out = {}
    for m in re.finditer(r"\b(\w+3D)\s*(?:\[\d+\])?\s*=\s*(\{[^}]*\}|[^,;{}]+)", text):
        name, value = m.group(1), m.group(2).strip()
        try:
            out[name] = [number(v) for v in value.strip("{}").split(",")] if value.startswith("{") else number(value)
        except ValueError:
            continue
    return out


def struct_body(text: str, name: str) -> str:
    start = text.index("struct " + name + " {")
    return text[start:text.index("\n};", start)]


def main(root: str) -> None:
    palettes_text = open(os.path.join(root, "Main_header", "WavePalettes.h")).read()
    table = palettes_text[palettes_text.index("palettes[]={"):palettes_text.index("};", palettes_text.index("palettes[]={"))]
    rows = re.findall(r"\{\{\{(.*?)\}\}\}", table)
    palettes = []
    for row in rows:
        stops = [[number(v) for v in stop.split(",")] for stop in row.split("},{")]
        palettes.append(stops)
    assert len(palettes) == 14 and all(len(p) == 5 for p in palettes)

    sim = open(os.path.join(root, "include", "Seis3D_Sim.h")).read()
    state = initialisers(struct_body(sim, "Seis3D_State"))
    camera = initialisers(struct_body(sim, "VolumeCamera3D"))
    defaults = {k: state[k] for k in STATE_FIELDS}
    defaults.update({k: camera[k] for k in CAMERA_FIELDS})

    common = open(os.path.join(root, "include", "Common3D.h")).read()
    limits = {k: int(re.search(r"constexpr int " + k + r"\s*=\s*(\d+)", common).group(1))
              for k in ("maxVolumeAxis3D", "maxVolumeOutput3D")}

    out = {"palettes": palettes, "state_defaults": defaults, "limits": limits,
           "source": "Main_header/WavePalettes.h, include/Seis3D_Sim.h, include/Common3D.h"}
    with open(os.path.join(HERE, "display_reference.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
