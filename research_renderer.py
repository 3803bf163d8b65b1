#!/usr/bin/env python
"""Headless launcher with the reference's command-line surface
(research_renderer.py:53-78): the same options drive the CUDA passes of
research_b200 instead of the Vulkan application.

    python research_renderer.py --frames 64 --screenshot out/cornell.png
    python research_renderer.py --pass restir_di --denoise --frames 8 --screenshot out/di.png
    python research_renderer.py procedural --frames 16 --screenshot out/room.png
    python research_renderer.py scene.glb --pass restir_di --pass restir_pt --frames 8

The optional scene argument is "cornell" (default), "procedural" (the seeded
1M-triangle room) or the path of a .gltf / .glb file (a file that fails to
load falls back to the Cornell box, as the reference does). There is no
window: --no-input is accepted for compatibility and --frames defaults to 1.
"""
import argparse
import sys


def _parse_args(argv):
    p = argparse.ArgumentParser(prog="research_renderer.py",
                                description="Research Renderer light-transport passes on a B200 (headless).")
    p.add_argument("scene", nargs="?", default="cornell", help="cornell | procedural | path to .gltf/.glb")
    p.add_argument("--pass", dest="passes", action="append", default=[], metavar="NAME",
                   choices=["restir_di", "restir_gi", "restir_pt"],
                   help="Enable a pass (repeatable).")
    p.add_argument("--denoise", action="store_true", help="Enable the A-trous denoiser.")
    p.add_argument("--exposure", type=float, default=None, metavar="X", help="Set tonemap exposure.")
    p.add_argument("--no-input", action="store_true", help="Accepted for compatibility (no window here).")
    p.add_argument("--frames", type=int, default=1, metavar="N", help="Render exactly N frames.")
    p.add_argument("--screenshot", default=None, metavar="PATH", help="Save a PNG of the final frame.")
    p.add_argument("--size", default="1280x720", metavar="WxH", help="Image size (the reference uses the window).")
    return p.parse_args(argv)


def main(argv=None):
    args = _parse_args(sys.argv[1:] if argv is None else argv)
    from research_b200.passes import Application

    w, h = (int(x) for x in args.size.lower().split("x"))
    app = Application()
    app.initialize(w, h)
    if args.scene == "procedural":
        app.load_procedural()
    elif args.scene.lower().endswith((".gltf", ".glb")):
        app.load_gltf(args.scene)
    elif args.scene != "cornell":
        raise SystemExit(f"unsupported scene '{args.scene}' (cornell | procedural | .gltf/.glb path)")
    for name in args.passes:
        app.set_pass_enabled(name, True)
    if args.denoise:
        app.set_pass_enabled("denoise", True)
    if args.exposure is not None:
        app.set_exposure(args.exposure)
    for _ in range(args.frames):
        app.step()
    if args.screenshot:
        app.capture_screenshot(args.screenshot)
    print(f"[research_renderer] scene={app.scene_name} size={app.window_size} frames={args.frames} "
          f"spp={app.accumulate.accumulated_spp}")
    app.shutdown()
    return 0


if __name__ == "__main__":
    try:
        sys.exit(main())
    except KeyboardInterrupt:
        sys.exit(130)
    except Exception as exc:  # mirror main.cpp: log + non-zero exit
        print(f"Unhandled exception: {exc}", file=sys.stderr)
        sys.exit(1)
