"""dnlPython - DynELA's Python model API, solved on the B200 engine.

The names, arguments and behaviour follow the reference's SWIG module
(Sources/dnlPython/dnlPython.i over Sources/dnlFEM/DynELA.h:40-100 and the
classes it exposes), so that DynELA model scripts run unchanged:

    import dnlPython as dnl
    model = dnl.DynELA('Taylor')
    model.createNode(1, 0.0, 0.0, 0.0) ...
    model.setDefaultElement(dnl.Element.ElQua4NAx)
    model.createElement(1, 1, 2, 8, 7) ...
    ...
    model.solve()

Model building happens here, on the host, as in the reference; `solve()`
hands the model to the engine (include/dnlgpu.h) and writes the history files
at their save times.  There is no CPU solver behind this module: without the
engine library or a CUDA device `solve()` raises EngineUnavailable.

Scope of the mirror: the elements ElQua4NAx, ElQua4N2D and ElHex8N3D, the Johnson-Cook
law, BoundaryRestrain / BoundarySpeed (+ DiscreteFunction / RampFunction time
functions) and the other boundary types with the reference's behaviour on the
explicit path (no effect, or a stop for a constant displacement or force), the Explicit solver with the Courant and power-iteration time
steps, HistoryFile, and the VTK result files of DynELA::setSaveTimes (written
by the engine library: the fields are extracted at the nodes on the device).
SvgInterface is accepted and skipped.
"""
import math
import os
import sys

import numpy as np

from . import _abi

__all__ = ["DynELA", "NodeSet", "ElementSet", "Material", "JohnsonCookLaw", "BoundaryRestrain", "BoundarySpeed",
           "BoundaryDisplacement", "BoundaryForce", "BoundaryAcceleration", "BoundaryTemperature",
           "BoundaryConvection", "BoundaryFlux",
           "DiscreteFunction", "RampFunction", "Explicit", "HistoryFile", "Field", "Element", "Vec3D",
           "SvgInterface", "Parallel", "VtkInterface"]


class Vec3D:
    """Three components, read with v(i) or v[i] (Vec3D.h)."""

    def __init__(self, x=0.0, y=0.0, z=0.0):
        self._v = [float(x), float(y), float(z)]

    def __call__(self, i):
        return self._v[i]

    def __getitem__(self, i):
        return self._v[i]

    def __setitem__(self, i, v):
        self._v[i] = float(v)

    def __repr__(self):
        return "Vec3D(%g, %g, %g)" % tuple(self._v)


class Element:
    """Element type codes of DynELA::setDefaultElement (Element.h)."""
    ElGeneric = 0
    ElQua4NAx = _abi.ELQUA4NAX
    ElHex8N3D = _abi.ELHEX8N3D
    ElQua4N2D = _abi.ELQUA4N2D
    # families outside the accelerated path
    ElTri3N2D = 102
    ElTet4N3D = 103
    ElTet10N3D = 104


def _field_names():
    """Field codes and labels in the order of Field.h:46-79 / Field.C (vtkNames)."""
    names = []

    def vec(n):
        names.extend([n, n + "X", n + "Y", n + "Z"])

    def ten(n):
        names.extend([n] + [n + a + b for a in "XYZ" for b in "XYZ"])

    for n in ("coords", "disp", "dispInc", "speed", "speedInc"):
        vec(n)
    names.extend(["density", "gamma", "gammaCumulate", "internalEnergy", "inelasticEnergy", "kineticEnergy", "mass",
                  "plasticStrain", "plasticStrainRate", "pressure", "realTimeStep", "T", "timeStep", "vonMises",
                  "yieldStress"])
    for n in ("PlasticStrain", "PlasticStrainInc", "Strain", "StrainInc", "Stress"):
        ten(n)
    return names


class _FieldMeta(type):
    pass


class Field(metaclass=_FieldMeta):
    """Field codes (Field::FieldLabel); `Field.label(code)` gives the history-file name."""
    _names = _field_names()

    @classmethod
    def label(cls, code):
        n = cls._names[code]
        return "yield" if n == "yieldStress" else n


for _i, _n in enumerate(Field._names):
    setattr(Field, _n, _i)


class NodeSet:
    def __init__(self, name=None):
        self.name = name or "NodeSet"
        self.numbers = []

    def size(self):
        return len(self.numbers)


class ElementSet:
    def __init__(self, name=None):
        self.name = name or "ElementSet"
        self.numbers = []

    def size(self):
        return len(self.numbers)


class JohnsonCookLaw:
    def __init__(self, name=None):
        self.name = name
        self.A = self.B = self.C = self.n = self.m = 0.0
        self.depsp0, self.Tm, self.T0 = 1.0, 0.0, 0.0

    def setParameters(self, A, B, C, n, m, depsp0, Tm, T0):
        """JohnsonCookLaw::setParameters (JohnsonCookLaw.C:132-143)."""
        self.A, self.B, self.C, self.n, self.m = float(A), float(B), float(C), float(n), float(m)
        self.depsp0, self.Tm, self.T0 = float(depsp0), float(Tm), float(T0)


class Material:
    def __init__(self, name=None):
        self.name = name or "Material"
        self.youngModulus = 0.0
        self.poissonRatio = 0.0
        self.density = 0.0
        self.heatCapacity = 0.0
        self.taylorQuinney = 0.0
        self.T0 = 0.0
        self._law = None

    def setHardeningLaw(self, law):
        if not isinstance(law, JohnsonCookLaw):
            raise NotImplementedError("only the Johnson-Cook law is available on the accelerated path")
        self._law = law

    def getHardeningLaw(self):
        return self._law

    def _desc(self):
        if self._law is None:
            raise ValueError(f"material {self.name} has no hardening law")
        L = self._law
        return _abi.material(young=self.youngModulus, poisson=self.poissonRatio, density=self.density,
                             heat_capacity=self.heatCapacity, taylor_quinney=self.taylorQuinney, T0=self.T0,
                             A=L.A, B=L.B, C=L.C, n=L.n, m=L.m, depsp0=L.depsp0, Tm=L.Tm, Tref=L.T0)


class DiscreteFunction:
    """Piecewise-linear function of time (DiscreteFunction.C:96-213)."""

    def __init__(self, name=None):
        self.name = name
        self.x, self.y = [], []

    def add(self, x, y):
        self.x.append(float(x))
        self.y.append(float(y))
        order = np.argsort(self.x, kind="stable")
        self.x = [self.x[i] for i in order]
        self.y = [self.y[i] for i in order]

    def getValue(self, x):
        return float(np.interp(x, self.x, self.y))

    def _table(self, t0, t1):
        return np.array(self.x), np.array(self.y)


class RampFunction:
    """RampFunction (RampFunction.C:40-132); the engine evaluates it as a
    piecewise-linear table of 4,001 points over [min, max], zero outside."""
    Unknown, Linear, Sinus, Constant, Erf, Soft = 0, 1, 2, 3, 4, 5

    def __init__(self, name=None):
        self.name = name
        self.type = RampFunction.Unknown
        self.min = self.max = 0.0

    def setFunction(self, type_, vmin, vmax):
        self.type, self.min, self.max = int(type_), float(vmin), float(vmax)

    def getValue(self, x):
        if self.type == RampFunction.Unknown or x < self.min or x > self.max:
            return 0.0
        mm = self.max - self.min
        p = (x - self.min) / mm
        if self.type == RampFunction.Linear:
            return -2.0 / mm * p + 2.0 / mm
        if self.type == RampFunction.Sinus:
            return 1.0 / (1.0 - 2.0 / math.pi) / mm * (1.0 - math.sin(math.pi / 2 * p))
        if self.type == RampFunction.Constant:
            return 1.0 / mm
        if self.type == RampFunction.Erf:
            return math.exp(-(5 * p) ** 2) / (math.sqrt(math.pi) * mm / 10)
        if self.type == RampFunction.Soft:
            return 1 / mm * (math.pi * math.sin(math.pi * p) / 2)
        raise ValueError("unknown ramp type")

    def _table(self, t0, t1):
        xs = np.linspace(self.min, self.max, 4001)
        ys = np.array([self.getValue(x) for x in xs])
        lo, hi = min(t0, self.min) - 1.0, max(t1, self.max) + 1.0
        return np.concatenate([[lo], [np.nextafter(self.min, -np.inf)], xs, [np.nextafter(self.max, np.inf)], [hi]]), \
            np.concatenate([[0.0, 0.0], ys, [0.0, 0.0]])


class _Boundary:
    def __init__(self, name=None):
        self.name = name
        self.value = [0.0, 0.0, 0.0]
        self.function = None

    def setValue(self, x, y=None, z=None):
        if isinstance(x, Vec3D):
            self.value = [x(0), x(1), x(2)]
        else:
            self.value = [float(x), float(y), float(z)]

    def setFunction(self, f):
        """Boundary::setFunction (Boundary.C:75-79)."""
        self.function = f


class BoundaryRestrain(_Boundary):
    """Restrains the components whose value is > 0 (BoundaryRestrain.C:98-128)."""


class BoundarySpeed(_Boundary):
    """Imposes the non-zero speed components, optionally scaled by a time
    function (BoundarySpeed.C:139-206); as an initial condition, sets the whole
    speed vector (BoundarySpeed.C:63-73)."""


class BoundaryDisplacement(_Boundary):
    """Imposed displacement.  As an initial condition it does nothing
    (BoundaryDisplacement.C:62-65); as a constant condition the reference stops
    at the first increment with "not yet implemented"
    (BoundaryDisplacement.C:72-76), and so does solve() here."""
    _constant_error = "BoundaryDisplacement::applyConstantOnNewFields: not yet implemented"


class BoundaryForce(_Boundary):
    """Imposed nodal force.  As an initial condition it does nothing
    (BoundaryForce.C:61-65); as a constant condition the explicit solver reaches
    Boundary::applyConstantOnNewFields, which stops (Boundary.h:62), and so does
    solve() here."""
    _constant_error = "BoundaryForce: applyConstantOnNewFields is not provided (Boundary.h:62)"


class BoundaryAcceleration(_Boundary):
    """Imposed acceleration: accepted, with no effect as an initial or a
    constant condition (BoundaryAcceleration.C:54-70)."""


class BoundaryTemperature(_Boundary):
    """Imposed temperature: accepted, with no effect as an initial or a
    constant condition (BoundaryTemperature.C:73-93)."""

    def setValue(self, temperature):
        self.value = float(temperature)


class BoundaryConvection(_Boundary):
    """Convection (exchange coefficient, fluid temperature): accepted, with no
    effect as an initial or a constant condition (BoundaryConvection.C:85-103)."""

    def setValue(self, hc, Tf):
        self.value = (float(hc), float(Tf))


class BoundaryFlux(_Boundary):
    """Heat flux: accepted, with no effect as an initial or a constant
    condition (BoundaryFlux.C:73-95)."""

    def setValue(self, flux):
        self.value = float(flux)


class Explicit:
    """Chung-Hulbert explicit solver settings (Explicit.C, Solver.C)."""
    Courant = _abi.TS_COURANT
    PowerIteration = _abi.TS_POWER_ITERATION
    PowerIterationUnder = 2

    def __init__(self, name=None):
        self.name = name
        self.startTime, self.endTime = 0.0, 0.0
        self.timeStepMethod = _abi.TS_COURANT  # Solver.h:33 (TimeStepMethod = 0)
        self.computeTimeStepFrequency = 10     # configuration.dnl: ComputeTimeStepFrequency
        self.timeStepSafetyFactor = 0.9        # configuration.dnl: TimeStepSafetyFactor
        self.dissipation = 0.8182              # Explicit.h: defaultSpectralRadius

    def setTimes(self, start, end):
        self.startTime, self.endTime = float(start), float(end)

    def setTimeStepMethod(self, method):
        if method == Explicit.PowerIterationUnder:
            raise NotImplementedError("the under-integrated power iteration is not available on the GPU path")
        self.timeStepMethod = int(method)

    def setComputeTimeStepFrequency(self, f):
        self.computeTimeStepFrequency = int(f)

    def setTimeStepSafetyFactor(self, s):
        self.timeStepSafetyFactor = float(s)

    def setDissipation(self, rho):
        if not 0.0 <= rho <= 1.0:
            raise ValueError("dissipation value out of range [0.0, 1.0]")
        self.dissipation = float(rho)


class HistoryFile:
    """Time-history file (HistoryFile.C): node, element and global items,
    written when the time reaches the next save time."""

    def __init__(self, name=None):
        self.name = name or "HistoryFile"
        self.fileName = ""
        self.items = []  # (label, kind, target, ip, field)
        self.saveTime = 0.0
        self.startTime = self.nextTime = 0.0
        self.stopTime = -1.0
        self._f = None

    def setFileName(self, f):
        self.fileName = str(f)

    def setSaveTime(self, save, stop=None, start=None):
        if stop is None:
            self.startTime, self.nextTime, self.saveTime, self.stopTime = 0.0, 0.0, float(save), -1.0
        else:
            # HistoryFile::setSaveTime(startTime, stopTime, saveTime) (HistoryFile.C:140-148)
            self.startTime, self.stopTime, self.saveTime = float(save), float(stop), float(start)
            self.nextTime = self.startTime

    def add(self, a, b=None, c=None):
        if isinstance(a, NodeSet):
            field = b
            base = Field.label(field)
            for num in a.numbers:
                lab = base if len(a.numbers) == 1 else f"{base}_n{num}"
                self.items.append((lab, "node", num, None, field))
        elif isinstance(a, ElementSet):
            ip, field = (b, c) if c is not None else (0, b)
            base = Field.label(field) + (f"_{ip}" if ip > 0 else "")
            for num in a.numbers:
                lab = base if len(a.numbers) == 1 else f"{base}_e{num}"
                self.items.append((lab, "element", num, ip - 1, field))
        else:
            self.items.append((Field.label(a), "global", None, None, a))

    def _due(self, t):
        # HistoryFile::save (HistoryFile.C:292-317)
        if t > self.startTime and t < self.nextTime:
            return False
        return True


class Parallel:
    """Parallel::setCores is accepted; the GPU path does not use host threads."""

    def __init__(self):
        self.cores = 1

    def setCores(self, n):
        self.cores = int(n)


class SvgInterface:
    """SVG contour plots are written by the reference on the host; this mirror
    accepts the calls and writes nothing."""

    def __init__(self, name=None):
        self.name = name

    def setTitleDisplay(self, *a):
        pass

    def setLegendPosition(self, *a):
        pass

    def rotate(self, *a):
        pass

    def write(self, *a):
        pass


class Node:
    """A node as scripts see it after solve(): number, coords, disp (Node.h:35-149)."""

    def __init__(self, model, number):
        self._model = model
        self.number = number

    def _row(self, field):
        m = self._model
        if getattr(m, "_engine", None) is None:  # before solve(): the created node
            x = np.array(m._nodes[self.number], dtype=np.float64)
            return x if field == _abi.NODE_COORDS else np.zeros(3)
        return m._node_field(field)[m._node_index[self.number]]

    @property
    def coords(self):
        return Vec3D(*self._row(_abi.NODE_COORDS))

    @property
    def disp(self):
        return Vec3D(*self._row(_abi.NODE_DISP))

    @property
    def mass(self):
        return float(self._row(_abi.NODE_MASS)[0])


class VtkInterface:
    """The fields of the result files (VtkInterface, VtkInterface.C:224-278):
    initially those of the reference's settings file (VtkFields) that it
    recognises; addField / removeField take dnl.Field codes."""

    # Sources/dnlSettings/configuration.dnl VtkFields, as Field::getField reads them
    DEFAULT = ["Stress", "Strain", "PlasticStrain", "vonMises", "yield", "pressure", "plasticStrain",
               "plasticStrainRate", "gamma", "gammaCumulate", "speed"]

    def __init__(self, name=None):
        self.name = name or "VtkInterface::_noname_"
        self.fields = list(self.DEFAULT)

    def initFields(self):
        self.fields = list(self.DEFAULT)

    @staticmethod
    def _label(field):
        label = Field.label(field) if isinstance(field, int) else str(field)
        if label not in _abi.VTK_FIELDS:
            raise ValueError(f"field {label} cannot be written to a result file")
        return label

    def existField(self, field):
        label = self._label(field)
        return self.fields.index(label) if label in self.fields else -1

    def addField(self, field):
        label = self._label(field)
        if label not in self.fields:
            self.fields.append(label)

    def removeField(self, field):
        label = self._label(field)
        if label in self.fields:
            self.fields.remove(label)

    def getNumberOfFields(self):
        return len(self.fields)


class DynELA:
    """The model (DynELA.h:40-100)."""

    def __init__(self, name=None):
        self.name = name or "DynELA"
        self._nodes = {}      # number -> (x, y, z)
        self._elements = {}   # number -> (type, node numbers)
        self._default_element = Element.ElGeneric
        self._node_sets = []
        self._element_sets = []
        self._materials = []  # (material, element set)
        self._initial_bcs = []   # (boundary, node set)
        self._constant_bcs = []
        self._histories = []
        self.solver = None
        self.parallel = Parallel()
        # DynELA::setSaveTimes: start, end, increment (defaults of DynELA.h:36-39)
        self.saveTimes = (0.0, 0.0, 0.0)
        self.dataFile = VtkInterface()
        self._vtk_index = 0
        self._next_save = 0.0
        self.precision = _abi.PREC_MIXED if os.environ.get("DNL_PRECISION", "fp64") == "mixed" else _abi.PREC_FP64
        self.stress_method = _abi.STRESS_NEWTON
        self._engine = None
        self._cache = {}
        self._node_index = {}
        # history records kept on the device (False: the run stops at every save time)
        self._use_history_ring = True

    # ---- model building (DynELA.C:160-297, 380-476)
    def createNode(self, number, x, y=None, z=None):
        if isinstance(x, Vec3D):
            x, y, z = x(0), x(1), x(2)
        if number in self._nodes:
            raise ValueError(f"Node {number} already exists in the node list of this model")
        self._nodes[int(number)] = (float(x), float(y), float(z))
        return True

    def createElement(self, number, *nodes):
        if self._default_element == Element.ElGeneric:
            raise ValueError("Element type not set")
        if self._default_element not in (Element.ElQua4NAx, Element.ElHex8N3D, Element.ElQua4N2D):
            raise NotImplementedError("only ElQua4NAx, ElQua4N2D and ElHex8N3D are available on the accelerated path")
        npe = _abi.NODES_PER_ELEMENT[self._default_element]
        if len(nodes) != npe:
            raise ValueError(f"element {number}: {len(nodes)} nodes given, {npe} expected")
        if number in self._elements:
            raise ValueError(f"Element {number} already exists")
        self._elements[int(number)] = (self._default_element, tuple(int(n) for n in nodes))
        return True

    def setDefaultElement(self, type_):
        self._default_element = int(type_)

    def getNodesNumber(self):
        return len(self._nodes)

    def getElementsNumber(self):
        return len(self._elements)

    def add(self, obj, a=-1, b=-1, c=1):
        if isinstance(obj, NodeSet):
            self._add_range(obj, self._nodes, a, b, c, "Node")
            if obj not in self._node_sets:
                self._node_sets.append(obj)
        elif isinstance(obj, ElementSet):
            self._add_range(obj, self._elements, a, b, c, "Element")
            if obj not in self._element_sets:
                self._element_sets.append(obj)
        elif isinstance(obj, Material):
            if not isinstance(a, ElementSet):
                raise TypeError("add(Material, ElementSet)")
            self._materials.append((obj, a))
        elif isinstance(obj, Explicit):
            self.solver = obj
        elif isinstance(obj, HistoryFile):
            self._histories.append(obj)
        else:
            raise TypeError(f"cannot add {type(obj).__name__} to a model")

    @staticmethod
    def _add_range(s, table, start, end, inc, what):
        # Model::add(NodeSet/ElementSet, start, end, increment) (Model.C:181-233)
        if start == -1:
            return
        nums = [start] if end == -1 else range(start, end + 1, inc)
        for n in nums:
            if n not in table:
                raise ValueError(f"{what} {n} not exist in current grid and model")
            s.numbers.append(int(n))

    def addMaterial(self, material):
        pass

    def attachConstantBC(self, bc, nodeSet):
        self._constant_bcs.append((bc, nodeSet))

    def attachInitialBC(self, bc, nodeSet):
        self._initial_bcs.append((bc, nodeSet))

    def setSaveTimes(self, start, end, inc):
        """DynELA::setSaveTimes (DynELA.C:479-487): result files from `start`
        to `end` every `inc` (the next save time starts at `start`)."""
        self.saveTimes = (float(start), float(end), float(inc))
        self._next_save = float(start)

    def setStressComputation(self, method):
        """DynELA::setStressComputation (DynELA.C:1407-1431): "NewtonRaphson"
        or "Direct" (the one-step return of Element::computeStressDirect)."""
        if str(method) == "Direct":
            self.stress_method = _abi.STRESS_DIRECT
        elif str(method) == "NewtonRaphson":
            self.stress_method = _abi.STRESS_NEWTON
        else:
            raise ValueError(f"Unknown setStressComputation method : {method}")

    def setPrecision(self, precision):
        """Extension: 'fp64' (default, the reference's arithmetic) or 'mixed'
        (FP32 element math, FP64 positions, time and energy sums)."""
        self.precision = _abi.PREC_MIXED if precision == "mixed" else _abi.PREC_FP64

    def getNodeByNum(self, number):
        if number not in self._nodes:
            return None
        return Node(self, number)

    # ---- description handed to the engine
    def _description(self):
        if not self._elements:
            raise ValueError("the model has no element")
        if self.solver is None:
            raise ValueError("no solver attached to the model")
        types = {t for t, _ in self._elements.values()}
        if len(types) != 1:
            raise NotImplementedError("one element type per model")
        etype = types.pop()
        node_nums = sorted(self._nodes)  # the reference keeps its lists sorted by number (Model.C:67-96)
        index = {n: i for i, n in enumerate(node_nums)}
        elem_nums = sorted(self._elements)
        eindex = {n: i for i, n in enumerate(elem_nums)}
        coords = np.array([self._nodes[n] for n in node_nums], dtype=np.float64)
        conn = np.array([[index[k] for k in self._elements[e][1]] for e in elem_nums], dtype=np.int32)
        # materials: the last assignment of an element wins
        mats, emat = [], -np.ones(len(elem_nums), np.int32)
        for mat, es in self._materials:
            if mat not in mats:
                mats.append(mat)
            k = mats.index(mat)
            for e in es.numbers:
                emat[eindex[e]] = k
        if (emat < 0).any():
            raise ValueError("every element needs a material")
        nN = len(node_nums)
        v = np.zeros((nN, 3))
        bc = np.zeros((nN, 3), np.int8)
        bcv = np.zeros((nN, 3))
        bcf = -np.ones((nN, 3), np.int32)
        funcs, fidx = [], {}
        t0, t1 = self.solver.startTime, self.solver.endTime
        # initial speeds: initial list, then the constant list (BoundaryCondition.C:131-154)
        per_node_init = [[] for _ in range(nN)]
        per_node_const = [[] for _ in range(nN)]
        for b, ns in self._initial_bcs:
            for n in ns.numbers:
                per_node_init[index[n]].append(b)
        for b, ns in self._constant_bcs:
            # the explicit solver applies every constant condition of a node at
            # each increment (Explicit.C:478,526); the types that stop there stop here
            if getattr(b, "_constant_error", None) and len(ns.numbers):
                raise RuntimeError(b._constant_error)
            for n in ns.numbers:
                per_node_const[index[n]].append(b)
        for i in range(nN):
            for b in per_node_init[i] + per_node_const[i]:
                if isinstance(b, BoundarySpeed):
                    v[i] = b.value
            for b in per_node_const[i]:
                for c in range(3):
                    if isinstance(b, BoundaryRestrain) and b.value[c] > 0:
                        bc[i, c], bcv[i, c], bcf[i, c] = _abi.BC_RESTRAIN, 0.0, -1
                    elif isinstance(b, BoundarySpeed) and b.value[c] != 0.0:
                        bc[i, c], bcv[i, c] = _abi.BC_SPEED, b.value[c]
                        if b.function is not None:
                            key = id(b.function)
                            if key not in fidx:
                                fidx[key] = len(funcs)
                                funcs.append(b.function._table(t0, t1))
                            bcf[i, c] = fidx[key]
                        else:
                            bcf[i, c] = -1
        s = self.solver
        return _abi.ModelDesc(etype, coords, conn, [m._desc() for m in mats], elem_mat=emat, v_init=v, bc_code=bc,
                              bc_value=bcv, bc_func=bcf, functions=funcs, t_start=t0, t_end=t1,
                              ts_method=s.timeStepMethod, ts_freq=s.computeTimeStepFrequency,
                              ts_safety=s.timeStepSafetyFactor, rho_b=s.dissipation,
                              precision=self.precision, stress_method=self.stress_method,
                              # script meshes keep their createNode numbering unless
                              # renumbering at least halves the element span
                              node_order=_abi.ORDER_AUTO), node_nums, elem_nums

    # ---- solve (DynELA.C:727-773 -> Explicit::solve on the engine)
    def solve(self):
        desc, node_nums, elem_nums = self._description()
        self._node_index = {n: i for i, n in enumerate(node_nums)}
        self._elem_index = {n: i for i, n in enumerate(elem_nums)}
        self._npe = desc.nodes_per_element
        print(f"\nProcessing DynELA ... {len(elem_nums)} elements, {len(node_nums)} nodes on the B200 engine")
        eng = self._make_engine(desc)
        self._engine = eng
        self._cache = {}
        for h in self._histories:
            if not h.fileName:
                raise ValueError(f"No file name specified for object : {h.name}")
            h._f = open(h.fileName, "w")
            h._f.write("#DynELA FEM Code v. 4.0 history file\n#plotted :" + "".join(it[0] + " " for it in h.items)
                       + "\n")
        self._plan_items()
        self._write_histories(initial=True)
        # the history records of the increments are kept on the device and the
        # run does not stop at their save times (dnl_engine_set_history)
        ring = self._use_history_ring and 0 < len(self._histories) <= 64
        if ring:
            eng.set_history([(h.startTime, h.nextTime, h.saveTime) for h in self._histories], capacity=256)
        self._vtk_index = 0
        # the initial result file (DynELA::solve -> writeResultFile after initSolve, DynELA.C:745)
        self._write_result_file(prev=False)
        t_end = desc.t_end
        while True:
            c = eng.control()
            if c["done"] or c["time"] >= t_end:
                break
            t = c["time"]
            if (not ring and any(h.saveTime > 0 and h.nextTime <= t for h in self._histories)) or self._result_due(t):
                # an increment passed more than one save time: the reference writes
                # again after the next increment (its next time lags behind)
                eng.run(t_pause=t_end, max_incs=1)
            else:
                pauses = [] if ring else [h.nextTime for h in self._histories if h.saveTime > 0]
                if self._next_save <= self.saveTimes[1]:
                    pauses.append(self._next_save)
                eng.run(t_pause=min(pauses) if pauses else t_end)
            self._cache = {}
            if ring:
                self._write_history_records()
            else:
                self._write_histories()
            self._write_result_file(prev=True)
        c = eng.control()
        print(f"{self.name} inc={c['increment']} time={c['time']:8.4E} timeStep={c['time_step']:8.4E}")
        for h in self._histories:
            h._f.close()
            h._f = None
        # the final result file (DynELA::solve -> writeVTKFile, DynELA.C:770)
        self._write_vtk(prev=False)
        return True

    # ---- result files (DynELA::writeResultFile / writeVTKFile, DynELA.C:489-504, 688-711)
    def _result_due(self, t):
        return t >= self._next_save and t <= self.saveTimes[1]

    def _write_result_file(self, prev):
        """At the end of an increment (Explicit::endStep, before the field
        swap, hence the nodal increments, speeds and accelerations of before
        it: prev) or at the start: a file when the time has reached the next
        save time and not passed the last one; the next save time then moves
        on by one increment of save time."""
        if self._result_due(self._engine.control()["time"]):
            self._write_vtk(prev)
            self._next_save += self.saveTimes[2]

    def _write_vtk(self, prev):
        path = f"{self.name}{self._vtk_index:03d}.vtk"
        t = self._engine.control()["time"]
        self._engine.write_vtk(path, self.dataFile.fields, prev=prev)
        print(f"Write VTK result file: {path} at time {t:g} s")
        self._vtk_index += 1

    @staticmethod
    def _make_engine(desc):
        from .engine import Engine
        return Engine(desc).init()

    def _node_field(self, field):
        if field not in self._cache:
            self._cache[field] = self._engine.nodes(field)
        return self._cache[field]

    # ---- history items: selected on the device, one gather per save time
    _NODE_FIELDS = (("coords", _abi.NODE_COORDS), ("dispInc", _abi.NODE_U), ("disp", _abi.NODE_DISP),
                    ("speedInc", _abi.NODE_ACCEL), ("speed", _abi.NODE_SPEED))

    @classmethod
    def _node_item(cls, field):
        """(nodal field, component suffix) of a node history field."""
        name = Field._names[field]
        for base, f in cls._NODE_FIELDS:
            if name.startswith(base) and name[len(base):] in ("X", "Y", "Z", ""):
                return f, name[len(base):]
        if name == "mass":
            return _abi.NODE_MASS, "X"
        raise NotImplementedError(f"node field {name}")

    def _item_keys(self, kind, target, ip, field):
        if kind == "global":
            if field == Field.kineticEnergy:
                return [(_abi.ITEM_KINETIC, _abi.NODE_SPEED, 0), (_abi.ITEM_KINETIC, _abi.NODE_SPEED_PREV, 0)]
            return []
        if kind == "node":
            f = self._node_item(field)[0]
            keys = [(_abi.ITEM_NODE, f, self._node_index[target])]
            if f in _abi.NODE_PREV:
                keys.append((_abi.ITEM_NODE, _abi.NODE_PREV[f], self._node_index[target]))
            return keys
        e = self._elem_index[target]
        qs = range(e * self._npe, (e + 1) * self._npe) if ip < 0 else [e * self._npe + ip]
        return [(_abi.ITEM_POINT, 0, q) for q in qs]

    def _plan_items(self):
        """The engine items every history file needs (HistoryFile::save reads,
        HistoryFile.C:289-317), registered once; a save time then copies only
        their values from the device."""
        keys = []
        for h in self._histories:
            for _, kind, target, ip, field in h.items:
                for k in self._item_keys(kind, target, ip, field):
                    if k not in keys:
                        keys.append(k)
        self._item_list = keys
        self._item_off = {}
        off = 0
        for k in keys:
            self._item_off[k] = off
            off += _abi.ITEM_WIDTH[k[0]]
        if keys:
            self._engine.set_items(keys)

    def _gathered(self, key):
        if "items" not in self._cache:
            self._cache["items"] = self._engine.gather_items()
        o = self._item_off[key]
        return self._cache["items"][o:o + _abi.ITEM_WIDTH[key[0]]]

    def _item_value(self, kind, target, ip, field, rec=None):
        """An item's value now (rec None) or in a device record (dict of
        increment, time_step; the values are in self._cache["items"])."""
        eng = self._engine
        c = rec if rec is not None else eng.control()
        if kind == "global":
            if field in (Field.timeStep, Field.realTimeStep):
                return c["time_step"] if rec is not None else c["last_time_step"]
            if field == Field.kineticEnergy:
                # Model::getTotalKineticEnergy on field0, written before the swap (Explicit.C:539-552)
                f = _abi.NODE_SPEED_PREV if c["increment"] > 0 else _abi.NODE_SPEED
                return float(self._gathered((_abi.ITEM_KINETIC, f, 0))[0])
            return 0.0
        if kind == "node":
            f, suf = self._node_item(field)
            # inside the loop the reference writes before its field swap
            # (Explicit.C:539-552): field0 is then the start of the increment
            if f in _abi.NODE_PREV and c["increment"] > 0:
                f = _abi.NODE_PREV[f]
            row = self._gathered((_abi.ITEM_NODE, f, self._node_index[target]))
            return float(np.linalg.norm(row)) if suf == "" else float(row["XYZ".index(suf)])
        return float(np.mean([self._ip_value(self._gathered(k), field)
                              for k in self._item_keys(kind, target, ip, field)]))

    @staticmethod
    def _ip_value(s, field):
        # Element::getIntPointValueExtract (Element.C:1195-1240)
        name = Field._names[field]
        scal = {"plasticStrain": _abi.IP_EPSP, "plasticStrainRate": _abi.IP_DEPSP, "gamma": _abi.IP_GAMMA,
                "gammaCumulate": _abi.IP_GAMMA_CUM, "yieldStress": _abi.IP_YIELD, "T": _abi.IP_T,
                "density": _abi.IP_DENSITY, "pressure": _abi.IP_PRESSURE, "internalEnergy": _abi.IP_EINT,
                "inelasticEnergy": _abi.IP_EINEL}
        if name in scal:
            return s[scal[name]]
        if name == "vonMises":
            xx, xy, xz, yy, yz, zz = s[0:6]
            return math.sqrt(((xx - yy) ** 2 + (yy - zz) ** 2 + (zz - xx) ** 2 + 6 * (xy * xy + yz * yz + xz * xz))
                             / 2.0)
        for base, off in (("PlasticStrain", _abi.IP_PLASTIC_STRAIN), ("Strain", _abi.IP_STRAIN),
                          ("Stress", _abi.IP_STRESS)):
            if name.startswith(base) and not name.startswith(base + "Inc"):
                t = s[off:off + 6]
                suf = name[len(base):]
                if suf == "":
                    return math.sqrt(t[0] ** 2 + t[3] ** 2 + t[5] ** 2 + 2 * (t[1] ** 2 + t[2] ** 2 + t[4] ** 2))
                i, j = "XYZ".index(suf[0]), "XYZ".index(suf[1])
                sym = [[0, 1, 2], [1, 3, 4], [2, 4, 5]]
                return t[sym[i][j]]
        raise NotImplementedError(f"point field {name}")

    def _write_history_records(self):
        """The lines of the records the device kept since the last look: for
        each record, every file whose schedule was due (its bit in the mask)."""
        for t, inc, dt, mask, values in self._engine.history_records():
            self._cache = {"items": values}
            rec = {"increment": inc, "time_step": dt}
            for j, h in enumerate(self._histories):
                if not (mask >> j) & 1:
                    continue
                h.nextTime += h.saveTime
                vals = [self._item_value(kind, target, ip, field, rec) for _, kind, target, ip, field in h.items]
                h._f.write("%10.7E " % t + "".join("%10.7E " % x for x in vals) + "\n")
            self._cache = {}
        for h in self._histories:
            h._f.flush()

    def _write_histories(self, initial=False):
        t = self._engine.control()["time"]
        for h in self._histories:
            if not h._due(t):
                continue
            h.nextTime += h.saveTime
            vals = [self._item_value(kind, target, ip, field) for _, kind, target, ip, field in h.items]
            h._f.write("%10.7E " % t + "".join("%10.7E " % x for x in vals) + "\n")
            h._f.flush()
