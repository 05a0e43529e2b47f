"""The stage classes (GPUImage, ImageModel, ImagePyramid, FlowPropagator, FlowPropagatorPayload,
FlowUpdate, DeltaFlowUpdate, FlowSmoother) wired into whole filters the way the reference wires
its own (src/gpu/flowfilter.cu:84-197, 371-503, 650-716), run on the reference parity
sequences and compared bit for bit with the reference library's flows."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import golden_case
from make_reference_fixtures import CASES, case_frames, sha

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sc(cuda):
    from flowfilter_b200 import stage_classes

    return stage_classes


def f32(x):
    return float(np.float32(x))


class Level:
    """FlowFilter (top = True) or DeltaFlowFilter built from stages."""

    def __init__(self, sc, image, coarse=None, top=True):
        self.top = top
        self.model = sc.ImageModel(image)
        h, w = image.height, image.width
        if top:
            dummy = sc.GPUImage((h, w, 2), 4)
            self.update = sc.FlowUpdate(dummy, self.model.getImageConstant(), self.model.getImageGradient(), 1.0,
                                        1.0)
            self.smoother = sc.FlowSmoother(self.update.getUpdatedFlow(), 1)
            self.prop = sc.FlowPropagator(self.smoother.getSmoothedFlow(), 1)
            self.update.setInputFlow(self.prop.getPropagatedFlow())
        else:
            dd, do = sc.GPUImage((h, w, 2), 4), sc.GPUImage((h, w), 4)
            self.update = sc.DeltaFlowUpdate(coarse, dd, do, self.model.getImageConstant(),
                                             self.model.getImageGradient())
            self.smoother = sc.FlowSmoother(self.update.getUpdatedFlow(), 1)
            self.prop = sc.FlowPropagatorPayload(self.smoother.getSmoothedFlow(), self.update.getUpdatedImage(),
                                                 self.update.getUpdatedDeltaFlow())
            self.update.setInputDeltaFlow(self.prop.getPropagatedVector())
            self.update.setInputImageOld(self.prop.getPropagatedScalar())
        self.first = True

    def set_params(self, gamma, smooth, maxflow, u8=True):
        self.update.gamma = f32(np.float32(gamma) / np.float32(255.0 * 255.0)) if u8 else gamma
        self.update.maxflow = maxflow
        self.prop.iterations = int(np.ceil(np.float32(maxflow)))
        self.smoother.iterations = smooth

    def flow(self):
        """getFlow(): the update's flow on the top level, the smoothed flow below."""
        return self.update.getUpdatedFlow() if self.top else self.smoother.getSmoothedFlow()

    def compute(self):
        self.model.compute()
        if self.first:
            self.update.getUpdatedImage().copyFrom(self.model.getImageConstant())
            self.first = False
        self.prop.compute()
        self.update.compute()
        self.smoother.compute()

    def compute_update(self):
        if self.first:
            a0 = self.model.getImageConstant()
            self.update.getUpdatedImage().copyFrom(a0)
            if not self.top:
                self.prop.getPropagatedScalar().copyFrom(a0)
            self.first = False
        self.update.compute()
        self.smoother.compute()


class StagePyramid:
    def __init__(self, sc, h, w, levels, gammas, smooths, maxflow):
        self.input = sc.GPUImage((h, w), 1)
        self.pyr = sc.ImagePyramid(self.input, max(levels, 1))
        L = max(levels, 1)
        self.top = Level(sc, self.pyr.getImage(L - 1))
        self.low = [None] * (L - 1)
        coarse = self.top.flow()
        for l in range(L - 2, -1, -1):
            self.low[l] = Level(sc, self.pyr.getImage(l), coarse, top=False)
            coarse = self.low[l].flow()
        m = np.float32(maxflow)
        for l in range(L - 1):
            self.low[l].set_params(gammas[l], smooths[l], f32(m))
            m = m / np.float32(2.0)
        self.top.set_params(gammas[L - 1], smooths[L - 1], f32(m))
        self.L = L

    def compute(self, frame):
        self.input.upload(frame)
        self.pyr.compute()
        if self.L == 1:
            self.top.compute()
            return
        self.top.model.compute()
        self.top.prop.compute()
        for lv in self.low:
            lv.model.compute()
            lv.prop.compute()
        self.top.compute_update()
        for lv in self.low:
            lv.compute_update()

    def smoothed_flow(self):
        lv = self.low[0] if self.L > 1 else self.top
        return lv.smoother.getSmoothedFlow().download()


@pytest.mark.parametrize("name", ["constant_320x240_L1", "odd_77x61_L1", "small_96x64_L2", "odd_150x98_L3"])
def test_stage_classes_rebuild_the_reference_filters(sc, name):
    case = CASES[name]
    meta, arr = golden_case(name)
    frames = case_frames(case)
    assert sha(frames) == meta["frames_sha256"]
    h, w = frames.shape[1:]
    f = StagePyramid(sc, h, w, case["levels"], case["gamma"], case["smooth"], case["maxflow"])
    got = []
    for t in range(frames.shape[0]):
        f.compute(frames[t])
        if t in case["dump"]:
            got.append(f.smoothed_flow())
    got = np.stack(got)
    if meta["layout"] == "full":
        assert np.max(np.abs(got - arr["flow"])) <= 1e-4
    assert [sha(x) for x in got] == meta["flow_sha256"]


def test_stage_outputs_are_shared_handles(sc, cuda):
    """Getters return the stage's own buffers, overwritten in place by every compute()."""
    rng = np.random.default_rng(3)
    img = sc.GPUImage((40, 56), 1)
    img.upload(rng.integers(0, 256, (40, 56), dtype=np.uint8))
    model = sc.ImageModel(img)
    a0 = model.getImageConstant()
    assert model.getImageConstant() is a0
    model.compute()
    ra0, rg = O.image_model(img.download())
    assert a0.download().tobytes() == ra0.tobytes()
    assert model.getImageGradient().download().tobytes() == rg.tobytes()
    img.upload(rng.integers(0, 256, (40, 56), dtype=np.uint8))
    model.compute()
    assert a0.download().tobytes() == O.image_model(img.download())[0].tobytes()
    assert model.elapsedTime() >= 0.0
    pyr = sc.ImagePyramid(img, 3)
    assert pyr.getImage(0) is img
    pyr.compute()
    assert pyr.getImage(2).download().tobytes() == O.pyramid_down(O.pyramid_down(img.download())).tobytes()
    flow = sc.GPUImage((40, 56, 2), 4)
    flow.upload(rng.normal(0, 1.5, (40, 56, 2)).astype(np.float32))
    p = sc.FlowPropagator(flow, 3)
    p.border = 2
    p.invertInputFlow = True
    p.compute()
    want = O.propagate(-flow.download(), 3, 2)
    assert p.getPropagatedFlow().download().tobytes() == want.tobytes()
    s = sc.FlowSmoother(p.getPropagatedFlow(), 2)
    s.compute()
    assert s.getSmoothedFlow().download().tobytes() == O.smooth(want, 2).tobytes()
    assert p.dt == float(np.float32(1) / np.float32(3))


def test_stage_argument_errors(sc, cuda):
    with pytest.raises(ValueError):
        sc.GPUImage((4,), 4)
    with pytest.raises(ValueError):
        sc.FlowUpdate().gamma = 0.0
    with pytest.raises(ValueError):
        sc.FlowSmoother(iterations=0)
    with pytest.raises(ValueError):
        sc.FlowPropagator(sc.GPUImage((4, 4), 4))  # depth 1 is not a flow
    with pytest.raises(RuntimeError):
        sc.ImageModel().compute()
    with pytest.raises(IndexError):
        sc.ImagePyramid(sc.GPUImage((8, 8), 1), 2).getImage(2)
    with pytest.raises(ValueError):
        sc.FlowPropagatorPayload(sc.GPUImage((8, 8, 2), 4), sc.GPUImage((8, 6), 4), sc.GPUImage((8, 8, 2), 4))
