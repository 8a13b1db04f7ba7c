"""Write tests/golden/scenes.json from the reference's own scene files.

The single-domain scenes this path runs are read as they stand in the reference
(crates/pantometry-world/scenes/*.json) and kept with the name of the file each came from, so the
scene tests load the reference's inputs rather than a retyping of them. Run from the repository
root with the reference checked out:

    python tests/golden/make_scenes.py /path/to/pantometry
"""
import json
import os
import sys

SCENES = {
    "room_mode": "01-room-mode.json",
    "room_higher_mode": "02-room-higher-mode.json",
    "room_pulse": "03-room-pulse.json",
    "block": "15-a-hot-spot-in-a-block.json",
    "hall": "16-a-room-with-a-ceiling.json",
    "block_meets_glass": "19-a-coating-stops-the-heat.json",
    "cavity": "27-a-cavity-ringing-at-its-own-frequency.json",
}


def main(root):
    base = os.path.join(root, "crates", "pantometry-world", "scenes")
    out = {}
    for key, name in SCENES.items():
        with open(os.path.join(base, name)) as f:
            out[key] = {"source": f"crates/pantometry-world/scenes/{name}", "scene": json.load(f)}
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "scenes.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
