"""HPCsharp's radix-sort extension methods, with the same names, argument meaning and
exceptions, running on the B200 through the C ABI (libhpcs_gpu.so).

Reference surface (paths relative to the HPCsharp project root):
  ParallelAlgorithm.SortRadixPar(this uint[], int ParallelWorkQuantum)  RadixSortLsdParallel.cs:145
  ParallelAlgorithm.SortRadixPar(this int[] / long[] / ulong[])         RadixSortLsdParallel.cs:446, :560, :690
  ParallelAlgorithm.SortRadixInPlaceInterfacePar(this T[])              RadixSortLsdParallel.cs:240, :677, :743
  Algorithm.SortRadixLsd(this T[] [, int start, int length])           RadixSortLsd.cs:255, :352, :437, :527
  Algorithm.SortRadixLsdFunc(this T[] [, int start, int length])       RadixSortLsd.cs:238, :315, :400, :490
  Algorithm.SortRadix(this uint[]) (examples' spelling, Program.cs:26)
  Algorithm.SortRadix<T>(this T[] items, UInt32[]/UInt64[] keys)        RadixSortLsd.cs:1183, :1245
  Algorithm.HistogramByteComponents(T[], int l, int r)                 Histogram.cs:261, :957, :992, :1019
  ParallelAlgorithm.HistogramByteComponentsPar(T[], int l, int r, ...)  HistogramParallel.cs:214, :416, :547, :617
  Algorithm.SelectTopK(this uint[], int k) / (a, start, length, k)     SelectionTopKRadix.cs:160, :142

Arrays are numpy arrays sorted in place (the reference's SortRadixPar returns the caller's
array after an even number of passes, RadixSortLsdParallel.cs:227-231).  float32/float64
keys are accepted too and ordered by the reference's float transform.
"""
from __future__ import annotations

import numpy as np

from .native import (ArgumentNullException, ArgumentOutOfRangeException, HPCS_ERR_NULL, HPCS_ERR_RANGE,
                     default_context)


def _require(a, name: str = "inputArray"):
    if a is None:
        raise ArgumentNullException(HPCS_ERR_NULL, f"{name} is null")


def SortRadixPar(inputArray: np.ndarray, ParallelWorkQuantum: int = 64 * 1024) -> np.ndarray:
    """Stable ascending LSD radix sort, in place; returns the caller's array.  The work
    quantum is the reference's CPU task size and has no effect on the GPU."""
    _require(inputArray)
    return default_context().sort(inputArray)


def SortRadixInPlaceInterfacePar(inputArray: np.ndarray) -> None:
    _require(inputArray)
    default_context().sort(inputArray)


def SortRadixLsd(inOutArray: np.ndarray, startIndex: int | None = None, length: int | None = None) -> None:
    """In-place serial-API sort; with (startIndex, length) sorts that subrange in place.
    (The reference's subrange overload writes its result to [0, length) because
    ComputeStartOfBins starts every bin at 0, RadixSortLsd.cs:120; this sorts the
    subrange where it lies.)"""
    _require(inOutArray, "inOutArray")
    if startIndex is None:
        default_context().sort(inOutArray)
        return
    if length is None or startIndex < 0 or length < 0 or startIndex + length > inOutArray.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "startIndex/length outside the array")
    default_context().sort(inOutArray[startIndex:startIndex + length])


def SortRadixLsdFunc(inOutArray: np.ndarray, startIndex: int | None = None, length: int | None = None):
    SortRadixLsd(inOutArray, startIndex, length)
    return inOutArray


def SortRadix(inputArray: np.ndarray, inKeys: np.ndarray | None = None):
    """SortRadix(this uint[]) sorts keys in place and returns them.
    SortRadix<T>(this T[] items, keys) sorts items by keys (stable), permuting both caller
    arrays in place, and returns (items, keys)."""
    if inKeys is None:
        _require(inputArray)
        return default_context().sort(inputArray)
    _require(inputArray)
    _require(inKeys, "inKeys")
    if inputArray.size != inKeys.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "items and keys differ in length")
    items = inputArray.view(np.uint32) if inputArray.dtype.itemsize == 4 else None
    if items is None:
        raise TypeError("items must be a 4-byte type (index payload)")
    default_context().sort_pairs(inKeys, items)
    return inputArray, inKeys


def HistogramByteComponentsPar(inArray: np.ndarray, l: int, r: int, parallelThreshold: int = 16 * 1024):
    """uint[P][256] digit counts of inArray[l..r] (inclusive)."""
    _require(inArray, "inArray")
    if l < 0 or r >= inArray.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "l/r outside the array")
    return default_context().histogram(inArray, l, r)


def HistogramByteComponents(inArray: np.ndarray, l: int, r: int):
    """int[P][256] digit counts of inArray[l..r] (inclusive)."""
    return HistogramByteComponentsPar(inArray, l, r).astype(np.int32)


def SelectTopK(arrayToBeSelected: np.ndarray, *args) -> None:
    """SelectTopK(a, k) or SelectTopK(a, start, length, k) (SelectionTopKRadix.cs:142-171),
    in place: afterwards a[k] is the k-th smallest and a[k..] the largest of the (sub)array.
    In the (start, length, k) form k indexes the whole array, as in the reference."""
    _require(arrayToBeSelected, "arrayToBeSelected")
    a = arrayToBeSelected
    if len(args) == 1:
        k = args[0]
        if a.size <= 0 or k < 0 or k >= a.size:
            raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
        default_context().select_topk(a, k)
        return
    start, length, k = args
    if start < 0 or length <= 0 or start + length > a.size:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "l or r are invalid")
    if k < start or k >= start + length:
        raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "k must be between start and (start + length)")
    default_context().select_topk(a[start:start + length], k - start)
